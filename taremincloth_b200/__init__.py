"""B200-native XPBD cloth substep (the hot path of Taremin/TareminCloth's cloth_core).

``ClothSimulator`` mirrors the reference's ``taremin_cloth_core.ClothSimulator``;
all computation runs in the in-tree CUDA library ``libtcloth.so``.
"""
from .simulator import BatchedClothSimulator, ClothSimulator, get_gpu_device_name, is_gpu_available  # noqa: F401

__all__ = ["ClothSimulator", "BatchedClothSimulator", "is_gpu_available", "get_gpu_device_name"]
