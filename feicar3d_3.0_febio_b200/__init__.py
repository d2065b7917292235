"""B200-native FEICAR3D pressure-Poisson path (tagging, ghost-cell BC,
multigrid) behind the reference's solver interface.  The directory name is
not a Python identifier; load it with :func:`load_package` (or import it as
``feicar_b200`` once loaded)."""
