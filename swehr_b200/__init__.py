"""B200-native SWEHR time step: CUDA kernels for sm_100a behind a C ABI
(include/swehr.h, libswehr.so), with Python host helpers for the
reference's input/output files and seeded synthetic workloads."""
