"""indicatrix_b200: a B200-native (sm_100a) CUDA backend for indicatrix's Path-Traced
spectral sample loop, behind a C ABI that mirrors the reference's ``GpuBackend``."""
