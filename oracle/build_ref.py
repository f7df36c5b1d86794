"""Build recipe for ``oracle/_ref``: the reference's own photon-differential splatting
extension, compiled unmodified from its two source files where they lie in the reference
checkout (``PyOptix/PhotonDifferentialSplattig.cpp`` and
``PyOptix/kernel/photon_differentials.cu``, with ``PyOptix/utils.hpp`` on the include
path). Nothing is copied: the sources are read in place and only build products are
written, into ``oracle/_ref/``.

This is test infrastructure. The built module is the reference's GPU kernel; it runs only
on a CUDA device and serves as (a) the generator of the golden fixtures under
``tests/golden/`` (via ``tests/golden/make_golden.py``) and (b) a parity check in the GPU
tests. The product never loads it.

The reference's own build (``setup.py``) also builds an OptiX module and needs the OptiX
SDK; that part is not built. This recipe calls ``torch.utils.cpp_extension.load`` on the two
splatting sources only, for sm_100 (``TORCH_CUDA_ARCH_LIST=10.0``), since the reference
carries no architecture flags of its own.

Usage: ``python oracle/build_ref.py [--ref-root PATH]``. The reference checkout is taken from
``--ref-root``, else from the ``PDS_REFERENCE_ROOT`` environment variable, else from
``/root/reference``; where none of these exists the recipe has nothing to build
(``reference_root()`` returns None).
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
MODULE = "pds_reference_ext"


DEFAULT_ROOT = "/root/reference"


def reference_root():
    """The reference checkout to build from, or None when it is not on this machine."""
    for cand in (os.environ.get("PDS_REFERENCE_ROOT"), DEFAULT_ROOT):
        if cand and os.path.isfile(os.path.join(cand, "PyOptix", "kernel",
                                                "photon_differentials.cu")):
            return cand
    return None


def built_path():
    """Path of the built reference module, or None if it has not been built."""
    build = os.path.join(OUT, "build")
    if not os.path.isdir(build):
        return None
    for f in os.listdir(build):
        if f.startswith(MODULE) and f.endswith(".so"):
            return os.path.join(build, f)
    return None


def build(ref_root=None, verbose=False):
    ref_root = ref_root or reference_root()
    if ref_root is None:
        raise FileNotFoundError("no reference checkout (set PDS_REFERENCE_ROOT)")
    srcs = [os.path.join(ref_root, "PyOptix", "PhotonDifferentialSplattig.cpp"),
            os.path.join(ref_root, "PyOptix", "kernel", "photon_differentials.cu")]
    for s in srcs:
        if not os.path.isfile(s):
            raise FileNotFoundError(s)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    os.makedirs(os.path.join(OUT, "build"), exist_ok=True)
    from torch.utils.cpp_extension import load
    load(name=MODULE, sources=srcs,
         extra_include_paths=[os.path.join(ref_root, "PyOptix")],
         build_directory=os.path.join(OUT, "build"), verbose=verbose)
    return built_path()


def load_module():
    """Import the built reference extension (requires torch; the kernels need a GPU)."""
    p = built_path()
    if p is None:
        raise ImportError("reference extension not built (run oracle/build_ref.py)")
    import importlib.util
    import torch  # noqa: F401  (the extension links against torch's libraries)
    spec = importlib.util.spec_from_file_location(MODULE, p)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=None)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.ref_root, a.verbose))
    sys.exit(0)
