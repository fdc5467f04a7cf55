"""celv2_b200: a B200-native decision engine for the CelV2 AV2 encoder.

The engine itself is CUDA (celv2_b200/csrc) behind a C ABI (include/celv2_cuda.h); this package
holds the Python mirror of the reference's DecisionEngine interface (``engine``), the build recipe
(``build``), the rate-weight table (``lam``) and the seeded synthetic clips (``synth``).
"""
