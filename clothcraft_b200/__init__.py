"""B200-native ClothCraft physics step: VBD colour sweeps + OGC contact on one GPU.

The compute path is the CUDA library ``clothcraft_b200/_lib/libclothcraft_b200.so``
(sm_100a) behind the C ABI in ``include/clothcraft.h``. This package holds the
Python host mirror of the reference's VbdSolver / OgcWorld interface and the
seeded scene generator. There is no CPU fallback: without the library the
solver classes raise.
"""
__all__ = ["abi", "scenes"]
