"""B200-native (sm_100a) single-GPU ECSIM particle cycle behind a C ABI.

tpic_b200/csrc holds the CUDA kernels and the C ABI (include/tpicb200.h);
`_lib` binds the built library, `simulation` drives the cycle, `plasma`
generates seeded synthetic plasmas and `deck` reads TPIC input decks.
"""
__all__ = ["_lib", "plasma", "simulation"]
