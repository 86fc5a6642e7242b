"""Drop-in module name of the reference's PyO3 extension (crates/cloth_py).

Re-exports the B200 implementation so code written against
``import taremin_cloth_core`` runs unchanged for the XPBD substep.
"""
from taremincloth_b200.simulator import ClothSimulator, get_gpu_device_name, is_gpu_available  # noqa: F401
