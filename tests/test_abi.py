"""CPU checks of the C ABI: the library exists, exports every entry point that
include/gpugrav.h declares, its struct layouts match the header, and argument
validation rejects bad parameters before any GPU work."""
import ctypes as C
import os
import subprocess
import tempfile

import pytest

from arepo_b200 import _lib as L
from arepo_b200 import build as B


@pytest.fixture(scope="module")
def lib():
    B.build()
    return L.load()


def test_header_declares_bound_symbols():
    declared = set(L.header_symbols())
    assert declared == set(L._SIGS), (declared ^ set(L._SIGS))


def test_library_exports_every_header_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = set(L.header_symbols()) - exported
    assert not missing, missing


def test_struct_layout_matches_header():
    src = r"""
#include <stddef.h>
#include <stdio.h>
#include "gpugrav.h"
int main(void){
 printf("%zu %zu %zu %zu %zu %zu\n", sizeof(gpugrav_params), sizeof(gpugrav_domain), sizeof(gpugrav_topnode),
        sizeof(gpugrav_tree_info), sizeof(gpugrav_timings), offsetof(gpugrav_params, precision));
 printf("%zu %zu %zu\n", offsetof(gpugrav_params, force_softening), offsetof(gpugrav_params, err_tol_theta),
        offsetof(gpugrav_topnode, morton_to_peano));
 return 0;}
"""
    with tempfile.TemporaryDirectory() as td:
        cpath, exe = os.path.join(td, "l.c"), os.path.join(td, "l")
        open(cpath, "w").write(src)
        subprocess.check_call(["gcc", "-I", os.path.dirname(L.HEADER), cpath, "-o", exe])
        a, b = subprocess.check_output([exe], text=True).splitlines()
    sizes = list(map(int, a.split()))
    offs = list(map(int, b.split()))
    assert sizes == [C.sizeof(L.Params), C.sizeof(L.Domain), L.TOPNODE_DTYPE.itemsize, C.sizeof(L.TreeInfo),
                     C.sizeof(L.Timings), L.Params.precision.offset]
    assert offs == [L.Params.force_softening.offset, L.Params.err_tol_theta.offset,
                    L.TOPNODE_DTYPE.fields["morton_to_peano"][1]]


def test_invalid_params_rejected_before_gpu_work(lib):
    ctx = C.c_void_p()
    p = L.make_params(periodic=True, asmth=0.01, rcut=0.0)  # the TreePM split needs Rcut > 0
    assert lib.gpugrav_create(C.byref(ctx), 0, C.byref(p)) == L.ERR_INVALID
    p = L.make_params(periodic=True, asmth=-0.01, rcut=0.04)  # Asmth < 0 (0 selects the Ewald-corrected tree)
    assert lib.gpugrav_create(C.byref(ctx), 0, C.byref(p)) == L.ERR_INVALID
    p = L.make_params(periodic=False)
    p.abi_version = 99
    assert lib.gpugrav_create(C.byref(ctx), 0, C.byref(p)) == L.ERR_INVALID
    p = L.make_params(periodic=False)
    p.force_softening[p.nsofttypes] = 1.0  # the trailing ForceSoftening entry must be 0
    assert lib.gpugrav_create(C.byref(ctx), 0, C.byref(p)) == L.ERR_INVALID
    assert lib.gpugrav_create(None, 0, C.byref(p)) == L.ERR_INVALID


def test_status_strings(lib):
    for s in (L.OK, L.ERR_TREE_FULL, L.ERR_TOPNODES, L.ERR_OUT_OF_BOX, L.ERR_INVALID, L.ERR_STATE):
        assert lib.gpugrav_status_string(s)
    assert b"-3" in lib.gpugrav_status_string(L.ERR_OUT_OF_BOX)


def test_null_context_calls_fail_cleanly(lib):
    assert lib.gpugrav_destroy(None) == L.ERR_INVALID
    assert lib.gpugrav_build(None, None, 0) == L.ERR_INVALID
    assert lib.gpugrav_walk(None, None, None, None, None, 0) == L.ERR_INVALID


def test_set_stream_handles():
    """GravityTree.set_stream: None asks for the context's own stream (NULL); torch's default stream
    (handle 0) is the legacy default stream, passed as cudaStreamLegacy so that the library's work is
    ordered after the caller's; other handles pass through.  A stand-in library records the calls."""
    import ctypes as C

    from arepo_b200.gravity import GravityTree

    seen = []

    class FakeLib:
        def gpugrav_set_stream(self, ctx, h):
            seen.append(None if h is None else h.value)
            return 0

    t = object.__new__(GravityTree)
    t.lib, t._ctx = FakeLib(), C.c_void_p(1)
    t._check = lambda s: None
    t.set_stream(None)
    t.set_stream(0)
    t.set_stream(0x7F00)
    assert seen == [None, 0x1, 0x7F00]
