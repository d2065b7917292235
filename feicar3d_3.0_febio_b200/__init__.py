"""B200-native FEICAR3D pressure-Poisson path (tagging, ghost-cell BC,
multigrid) behind the reference's solver interface.

The directory name is not a Python identifier, so the package is loaded
from its path under the name ``feicar_b200``::

    spec = importlib.util.spec_from_file_location(
        "feicar_b200", "<repo>/feicar3d_3.0_febio_b200/__init__.py",
        submodule_search_locations=["<repo>/feicar3d_3.0_febio_b200"])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["feicar_b200"] = mod
    spec.loader.exec_module(mod)
    from feicar_b200 import fg, synth

(``tests/conftest.py``, ``bench.py`` and ``__graft_entry__.py`` do this.)
"""
