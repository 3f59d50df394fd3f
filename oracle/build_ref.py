"""Build recipe for the reference PICT extension, used only as a test oracle.

This compiles the reference's own CUDA/C++ sources where they lie (the
``extensions/`` folder of the PICT checkout, read-only) into
``oracle/_ref/PISOtorch*.so``.  Nothing is copied into this repository: the
sources are passed to ``torch.utils.cpp_extension.load`` by absolute path and
only build products are written, into ``oracle/_ref/`` (git-ignored).

The resulting module is the reference's pybind11 ``PISOtorch`` and is used by
the ``tests/golden/make_ref_*.py`` scripts on a GPU machine to produce golden
fixtures that pin the CPU oracle (``oracle/piso_oracle.py``) and the CUDA path,
and by ``bench.py``'s reference timings.  It is never imported by the product
path (``pict_b200``).

Usage::

    python oracle/build_ref.py --src <PICT checkout>/extensions
    PICT_REF_EXTENSIONS=<PICT checkout>/extensions python oracle/build_ref.py

The source list and compiler flags follow the reference's extensions/setup.py:8-20
(same sources, ``-O3 --use_fast_math`` for nvcc, ``-Ofast`` for the host
compiler); the architecture is pinned to sm_100 for the B200.
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

# extensions/setup.py:8-11
REF_SOURCES = [
    "resampling.cu", "PISOtorch.cpp", "domain_structs.cpp", "PISO_multiblock_cuda_kernel.cu",
    "cg_solver_kernel.cu", "bicgstab_solver_kernel.cu", "grid_gen.cu",
    "eigenvalue.cu", "ortho_basis.cu", "matrix_vector_ops.cu", "matrix_vector_ops_grads.cu",
]


def build(src_dir, verbose=True):
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    from torch.utils import cpp_extension
    build_dir = os.path.join(OUT, "build")
    os.makedirs(build_dir, exist_ok=True)
    sources = [os.path.join(src_dir, s) for s in REF_SOURCES]
    for s in sources:
        if not os.path.isfile(s):
            raise FileNotFoundError(s)
    mod = cpp_extension.load(
        name="PISOtorch",
        sources=sources,
        extra_include_paths=[src_dir],
        extra_cflags=["-fvisibility=hidden", "-Ofast", "-DPYTHON_EXTENSION_BUILD=1"],
        extra_cuda_cflags=["-O3", "--use_fast_math", "-DPYTHON_EXTENSION_BUILD=1",
                           "-gencode", "arch=compute_100,code=sm_100"],
        extra_ldflags=["-L/usr/local/cuda/lib64", "-lcusparse", "-lcublas"],
        build_directory=build_dir,
        verbose=verbose,
        with_cuda=True,
    )
    # place the built module directly in oracle/_ref so it can be imported from there
    so = getattr(mod, "__file__", None)
    if so and os.path.dirname(os.path.abspath(so)) != OUT:
        import shutil
        shutil.copy2(so, os.path.join(OUT, os.path.basename(so)))
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=os.environ.get("PICT_REF_EXTENSIONS"),
                    help="the extensions/ folder of a PICT checkout (default: $PICT_REF_EXTENSIONS)")
    ap.add_argument("--quiet", action="store_true")
    args = ap.parse_args()
    if not args.src or not os.path.isdir(args.src):
        print("reference sources not given or not present (%s); nothing to build" % args.src)
        return 0
    build(args.src, verbose=not args.quiet)
    print("built reference extension into", OUT)
    return 0


if __name__ == "__main__":
    sys.exit(main())
