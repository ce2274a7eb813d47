"""vipe_b200 — B200-native (sm_100a) implementation of ViPE's DROID-style SLAM
backend hot path: dense bundle adjustment, correlation build/lookup and the
lietorch group kernels, behind the reference's slam_ext / droid_net_ext /
lietorch_ext Python entry points (see vipe_b200.ext)."""

__version__ = "0.1.0"
