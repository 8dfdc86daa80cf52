"""B200-native capsule contact mechanics for MicroSimulator.

The package holds the CUDA backend (``csrc/``, built in-tree into
``libmsb200.so``), its ctypes binding (``abi``), the host containers
(``world``), the parameter types (``types``), the backend and simulation
front ends (``backend``, ``simulation``) and the synthetic workloads
(``workloads``).
"""
