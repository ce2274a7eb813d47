// Test-only Python module around the reference's own correlation extension.
//
// The reference registers its droid_net_ext functions through
// `pybind_droid_net_ext(py::module&)` (csrc/droid_net_ext/droid.cpp:75-81) and
// builds every extension into one module (csrc/bind.cpp).  This file gives that
// one registration function a module of its own, so that the reference's
// correlation kernels (altcorr_kernel.cu, correlation_kernels.cu, droid.cpp),
// compiled unchanged from their sources by oracle/build_ref.py, can be loaded
// on the GPU box beside vipe_b200 and run on the same inputs.  It is part of
// the oracle: tests import it as the checker, the product never does.

#include <torch/extension.h>

void pybind_droid_net_ext(py::module& m);

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) { pybind_droid_net_ext(m); }
