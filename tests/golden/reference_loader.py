"""Load the reference's own rigid-contact source under the CPU Warp emulation -- TEST INFRASTRUCTURE.

warp-lang (the reference's runtime) is not installed in this image, so the reference cannot be
imported the normal way.  This loader puts ``tests/golden/warp_emulation`` on ``sys.path`` as the
``warp`` package and imports the reference's modules on the rigid-contact path
(``newton/_src/{core,math,geometry,sim,solvers}``) file by file from the reference tree, without
running the package ``__init__`` files (they pull in USD/MJCF importers, viewers and the other
solvers).  Modules that the path imports but never calls into (SDF, hydroelastic, heightfield,
contact reduction, sorting, matching, soft contacts) are replaced by placeholders that raise if
they are ever called.

Used only by ``tests/golden/make_golden.py``; the reference tree is read from the directory given
to :func:`load` (the script's ``--reference`` argument).
"""

from __future__ import annotations

import importlib
import importlib.util
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
EMULATION = os.path.join(HERE, "warp_emulation")

# modules on the import graph of the path whose code the path never runs
_PLACEHOLDER_MODULES = (
    "newton._src.geometry.sdf_contact",
    "newton._src.geometry.sdf_hydroelastic",
    "newton._src.geometry.sdf_texture",
    "newton._src.geometry.sdf_utils",
    "newton._src.geometry.contact_reduction_global",
    "newton._src.geometry.contact_reduction",
    "newton._src.geometry.contact_reduction_hydroelastic",
    "newton._src.geometry.contact_sort",
    "newton._src.geometry.contact_match",
    "newton._src.geometry.differentiable_contacts",
    "newton._src.geometry.kernels",
    "newton._src.geometry.broad_phase_sap",
    "newton._src.geometry.raycast",
    "newton._src.geometry.hashtable",
    "newton._src.geometry._sdf_cache",
    "newton._src.utils.heightfield",
    "newton._src.utils.texture",
    "newton._src.sim.model",
    "newton._src.sim.builder",
)


class _Placeholder(types.ModuleType):
    """A module whose every attribute is a placeholder class that raises when used."""

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        modname = self.__name__

        class _P:
            def __init__(self, *a, **k):
                raise NotImplementedError(f"{modname}.{name} is outside the emulated path")

            def __class_getitem__(cls, item):
                return cls

            def __call__(self, *a, **k):
                raise NotImplementedError(f"{modname}.{name} is outside the emulated path")

        _P.__name__ = name
        setattr(self, name, _P)
        return _P


def _package(name: str, path: str | None):
    m = types.ModuleType(name)
    m.__path__ = [path] if path else []
    m.__package__ = name
    sys.modules[name] = m
    return m


def _exec_module(name: str, path: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    # inside kernels ``float(x)`` is an fp32 conversion and ``float`` an fp32 annotation
    import warp

    mod.__dict__["float"] = warp.Float32Cast
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


class _Fp32Finder:
    """Meta-path finder for ``newton._src.*``: loads the reference's source files with ``float``
    bound to the fp32 conversion (see _exec_module)."""

    def __init__(self, root: str):
        self.root = root

    def find_spec(self, fullname, path=None, target=None):
        if not fullname.startswith("newton._src."):
            return None
        rel = fullname.split(".")[1:]
        base = os.path.join(self.root, *rel)
        if os.path.isfile(base + ".py"):
            return importlib.util.spec_from_file_location(fullname, base + ".py", loader=_Fp32Loader(base + ".py"))
        return None


class _Fp32Loader(importlib.abc.Loader if hasattr(importlib, "abc") else object):
    def __init__(self, path):
        self.path = path

    def create_module(self, spec):
        return None

    def exec_module(self, module):
        import warp

        module.__dict__["float"] = warp.Float32Cast
        code = compile(open(self.path).read(), self.path, "exec")
        exec(code, module.__dict__)


def load(reference_root: str):
    """Import the reference modules of the path; returns a namespace of them."""
    import importlib.abc  # noqa: F401

    if EMULATION not in sys.path:
        sys.path.insert(0, EMULATION)
    import warp

    if getattr(warp, "__version__", "") != "emulated":
        raise RuntimeError("a real warp package shadows the emulation")
    src = os.path.join(reference_root, "newton", "_src")
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference tree not found: {src}")
    for k in [k for k in sys.modules if k == "newton" or k.startswith("newton.")]:
        del sys.modules[k]
    _package("newton", os.path.join(reference_root, "newton"))
    _package("newton._src", src)
    for sub in ("core", "geometry", "sim", "solvers", "solvers.xpbd", "utils"):
        _package(f"newton._src.{sub}", os.path.join(src, *sub.split(".")))
    sys.meta_path.insert(0, _Fp32Finder(src))
    for name in _PLACEHOLDER_MODULES:
        sys.modules[name] = _Placeholder(name)

    class HydroelasticSDF:
        """No shape of these scenes is hydroelastic: the reference's _from_model returns None then
        (sdf_hydroelastic.py), which is all the pipeline asks of it."""

        Config = None

        @staticmethod
        def _from_model(model, config=None, writer_func=None):
            return None

    sys.modules["newton._src.geometry.sdf_hydroelastic"].HydroelasticSDF = HydroelasticSDF

    class ContactSorter:
        """Stand-in for contact_sort.ContactSorter (its radix sort is a Warp library routine): sorts
        the live contacts by their int64 key and gathers every per-contact array, which is what
        sort_full does (contact_sort.py:305-445; keys are unique per contact)."""

        def __init__(self, capacity, per_contact_shape_properties=False, device=None):
            self.capacity = capacity

        def sort_full(self, sort_keys, contact_count, device=None, **arrays):
            import numpy as np

            n = min(int(contact_count.numpy()[0]), self.capacity)
            order = np.argsort(sort_keys.numpy()[:n], kind="stable")
            sort_keys.data[:n] = sort_keys.data[:n][order]
            for a in arrays.values():
                if a is not None and a.data.size and a.shape[0] >= n:
                    a.data[:n] = a.data[:n][order]

    sys.modules["newton._src.geometry.contact_sort"].ContactSorter = ContactSorter

    # real modules: enums and flags first (package attributes other modules import)
    enums = importlib.import_module("newton._src.sim.enums")
    sim = sys.modules["newton._src.sim"]
    for k in ("BodyFlags", "JointType", "EqType"):
        if hasattr(enums, k):
            setattr(sim, k, getattr(enums, k))
    for k in ("Model", "ModelBuilder"):
        setattr(sim, k, type(k, (), {}))
    sim.Contacts = importlib.import_module("newton._src.sim.contacts").Contacts
    sim.State = importlib.import_module("newton._src.sim.state").State
    sim.Control = importlib.import_module("newton._src.sim.control").Control
    flags = importlib.import_module("newton._src.geometry.flags")
    geo = sys.modules["newton._src.geometry"]
    for k in ("ParticleFlags", "ShapeFlags"):
        if hasattr(flags, k):
            setattr(geo, k, getattr(flags, k))
    # the math package: its __init__ is the module the kernels import functions from
    math_pkg = os.path.join(src, "math")
    spec = importlib.util.spec_from_file_location("newton._src.math", os.path.join(math_pkg, "__init__.py"),
                                                  submodule_search_locations=[math_pkg],
                                                  loader=_Fp32Loader(os.path.join(math_pkg, "__init__.py")))
    mathmod = importlib.util.module_from_spec(spec)
    sys.modules["newton._src.math"] = mathmod
    spec.loader.exec_module(mathmod)

    ns = types.SimpleNamespace()
    ns.types = importlib.import_module("newton._src.geometry.types")
    ns.contact_data = importlib.import_module("newton._src.geometry.contact_data")
    ns.primitive = importlib.import_module("newton._src.geometry.collision_primitive")
    ns.support = importlib.import_module("newton._src.geometry.support_function")
    ns.core = importlib.import_module("newton._src.geometry.collision_core")
    ns.broad_common = importlib.import_module("newton._src.geometry.broad_phase_common")
    ns.narrow = importlib.import_module("newton._src.geometry.narrow_phase")
    ns.collide = importlib.import_module("newton._src.sim.collide")
    ns.xpbd_kernels = importlib.import_module("newton._src.solvers.xpbd.kernels")
    ns.solver = importlib.import_module("newton._src.solvers.solver")
    ns.solver_xpbd = importlib.import_module("newton._src.solvers.xpbd.solver_xpbd")
    ns.math = mathmod
    ns.warp = warp
    return ns
