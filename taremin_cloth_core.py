"""Drop-in module name of the reference's PyO3 extension (crates/cloth_py).

Re-exports the B200 implementation so code written against
``import taremin_cloth_core`` runs unchanged for the XPBD substep.
"""
from taremincloth_b200.simulator import (ClothSimulator, bake_bone_sdf_gpu, bake_mesh_sdf_coarse_gpu,  # noqa: F401
                                        bake_mesh_sdf_gpu, bake_mesh_sdf_hierarchical_gpu, color_edge_pairs,
                                        compute_areal_inv_masses, compute_combined_inv_masses,
                                        find_triangle_intersections,
                                        get_gpu_device_name, is_gpu_available)
