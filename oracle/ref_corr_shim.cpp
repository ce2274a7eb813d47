// Test-only Python module around the reference's own spatial-correlation
// extension (the AOT tracker's corr_ext).
//
// The reference registers it through `pybind_corr_ext(py::module&)`
// (csrc/corr_ext/correlation_sampler.cpp:82-85) inside its one combined module
// (csrc/bind.cpp).  This file gives that registration function a module of its
// own, so that the reference's CPU and CUDA correlation sampler, compiled
// unchanged from its sources by oracle/build_ref.py, can be run beside
// vipe_b200 on the same inputs.  It is part of the oracle: tests import it as
// the checker, the product never does.

#include <torch/extension.h>

void pybind_corr_ext(py::module& m);

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) { pybind_corr_ext(m); }
