"""CPU tests of the C ABI boundary: the CUDA library and the oracle load, and export every entry point the header declares."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "splashtank_cuda.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:[\w\*]+\s+)+\*?(st_\w+)\s*\(", txt, flags=re.M)))


def test_header_declares_the_flip_api():
    names = declared()
    for n in ("st_flip_create", "st_flip_step", "st_flip_read_particles", "st_flip_stats", "st_flip_destroy", "st_pbf_step"):
        assert n in names


def test_cuda_library_exports_every_declared_symbol():
    from splashtank_b200 import build
    path = build.build()
    lib = C.CDLL(path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, "not exported: %s" % missing
    lib.st_abi_version.restype = C.c_uint32
    assert lib.st_abi_version() == 1


def test_bindings_match_the_library():
    from splashtank_b200 import abi, build
    lib = C.CDLL(build.build())
    lists = (abi.FLIP_FUNCS + abi.CUDA_ONLY_FUNCS + abi.PBF_FUNCS + abi.POISSON_FUNCS + abi.NOALLOC_FUNCS + abi.BATCH_FUNCS + abi.DIFF_FUNCS +
             abi.SDF_FUNCS + abi.OCEAN_FUNCS)
    f = abi.bind(lib, "st_", lists)
    assert len(f) == len(lists)


def test_struct_sizes_match_the_header():
    """ctypes mirrors and the C structs agree (offsets of the last field and sizes), checked by compiling a probe."""
    import subprocess
    import tempfile
    from splashtank_b200 import abi
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "splashtank_cuda.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(st_flip_desc), sizeof(st_step_opts), sizeof(st_collider), sizeof(st_sdf),
         sizeof(st_stats), sizeof(st_flip_grid), sizeof(st_stage_times), sizeof(st_pbf_desc), sizeof(st_pbf_opts));
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(st_poisson_desc), sizeof(st_poisson_opts), sizeof(st_poisson_result), sizeof(st_poisson_system),
         sizeof(st_batch_desc), sizeof(st_diff_desc), sizeof(st_live_layout), sizeof(st_mesh), sizeof(st_sdf_build));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "p")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(x) for x in (abi.FlipDesc, abi.StepOpts, abi.Collider, abi.Sdf, abi.Stats, abi.Grid, abi.StageTimes, abi.PbfDesc, abi.PbfOpts,
                                  abi.PoissonDesc, abi.PoissonOpts, abi.PoissonResult, abi.PoissonSystem, abi.BatchDesc, abi.DiffDesc,
                                  abi.LiveLayout, abi.Mesh, abi.SdfBuild)]
    assert got == want


def test_product_path_has_no_cpu_fallback():
    """The product package never imports or loads the oracle; without the CUDA library it raises instead of computing."""
    import splashtank_b200
    pkg = os.path.dirname(splashtank_b200.__file__)
    for fn in os.listdir(pkg):
        if fn.endswith(".py"):
            src = open(os.path.join(pkg, fn)).read()
            assert not re.search(r"^\s*(from|import)\s+oracle", src, flags=re.M), fn
            assert "liboracle" not in src, fn
