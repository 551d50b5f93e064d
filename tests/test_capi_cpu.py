"""C-ABI boundary checks that need no GPU: the library loads, exports every
symbol include/rmetis.h declares, and answers host-side input errors with the
reference's codes (src/ffi/c_api.rs:157-167)."""
import ctypes
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT, greedy_options


def header_symbols():
    text = open(os.path.join(ROOT, "include", "rmetis.h")).read()
    return sorted(set(re.findall(r"RMETIS_API\s+(?:int|int64_t)\s+(RMETIS_\w+)\s*\(", text)))


def test_header_declares_drop_in_symbols():
    syms = header_symbols()
    assert "RMETIS_PartGraphKway" in syms and "RMETIS_SetDefaultOptions" in syms


def test_library_exports_every_header_symbol(rmb):
    lib = rmb._lib.load()
    for s in header_symbols():
        assert hasattr(lib, s), s
    assert set(header_symbols()) == set(rmb._lib.SIGNATURES)


def test_set_default_options_matches_reference(rmb, oracle):
    a = rmb.set_default_options()
    rc, b = oracle.set_default_options()
    assert rc == 1 and (a == b).all()


def test_set_default_options_null(rmb):
    assert rmb._lib.load().RMETIS_SetDefaultOptions(None) == -2


ENTRIES = ["RMETIS_PartGraphKway", "RMETIS_PartGraphRecursive"]  # c_api.rs:56-81 and :27-53


def _call(lib, n, ncon, xadj, adj, nparts, part, options=None, vwgt=None, adjwgt=None, null=(),
          entry="RMETIS_PartGraphKway"):
    I32P = ctypes.POINTER(ctypes.c_int32)
    nv = ctypes.c_int32(n); nc = ctypes.c_int32(ncon); npr = ctypes.c_int32(nparts)
    p = lambda a: None if a is None else np.ascontiguousarray(a, np.int32).ctypes.data_as(I32P)
    args = dict(nvtxs=ctypes.byref(nv), ncon=ctypes.byref(nc), xadj=p(xadj), adjncy=p(adj), vwgt=p(vwgt),
                vsize=None, adjwgt=p(adjwgt), nparts=ctypes.byref(npr), tpwgts=None, ubvec=None, options=p(options),
                objval=None, part=part.ctypes.data_as(I32P))
    for k in null:
        args[k] = None
    return getattr(lib, entry)(*args.values())


@pytest.mark.parametrize("entry", ENTRIES)
@pytest.mark.parametrize("missing", ["nvtxs", "ncon", "xadj", "adjncy", "nparts", "part"])
def test_null_required_pointer_is_input_error(rmb, missing, entry):
    xadj = np.array([0, 2, 4, 6, 8]); adj = np.array([1, 3, 0, 2, 1, 3, 0, 2])
    part = np.zeros(4, np.int32)
    assert _call(rmb._lib.load(), 4, 1, xadj, adj, 2, part, greedy_options(), null=(missing,), entry=entry) == -2


@pytest.mark.parametrize("entry", ENTRIES)
@pytest.mark.parametrize("n,ncon,nparts", [(0, 1, 2), (4, 0, 2), (4, 1, 1), (4, 1, -3)])
def test_scalar_input_errors(rmb, n, ncon, nparts, entry):
    xadj = np.array([0, 2, 4, 6, 8]); adj = np.array([1, 3, 0, 2, 1, 3, 0, 2])
    part = np.zeros(4, np.int32)
    assert _call(rmb._lib.load(), n, ncon, xadj, adj, nparts, part, greedy_options(), entry=entry) == -2


@pytest.mark.parametrize("entry", ENTRIES)
def test_bad_xadj0_is_input_error(rmb, entry):
    part = np.zeros(4, np.int32)
    assert _call(rmb._lib.load(), 4, 1, np.array([1, 2, 4, 6, 8]), np.array([1, 3, 0, 2, 1, 3, 0, 2]), 2, part,
                 greedy_options(), entry=entry) == -2


def test_options_codec_roundtrip(rmb):
    o = rmb.Options(ctype=rmb.CType.Rm, iptype=rmb.IpType.Random, rtype=rmb.RType.Greedy, ncuts=4, niter=7,
                    seed=99, ufactor=50)
    o2 = rmb.Options.from_raw(o.to_raw())
    assert o2 == o
    d = rmb.Options.from_raw(rmb.Options().to_raw())
    assert d == rmb.Options()


def test_python_validation_matches_oracle(rmb, oracle):
    cases = [
        (4, 1, [0, 2, 4, 6, 8], [1, 3, 0, 2, 1, 3, 0, 2], None),
        (4, 1, [0, 2, 4], [1, 3, 0, 2, 1, 3, 0, 2], None),
        (4, 1, [0, 3, 5, 7, 9], [0, 1, 3, 0, 2, 1, 3, 0, 2], None),
        (4, 1, [0, 1, 1, 0, 0], [1], None),
        (4, 1, [0, 2, 4, 6, 8], [1, 3, 0, 2, 1, 3, 0, 2], [1, 1, 1]),
        (4, 1, [0, 2, 4, 6, 8], [1, 3, 0, 2, 1, 3, 0, 2], [1, 0, 1, 1]),
    ]
    for n, ncon, x, a, vw in cases:
        want_ok = oracle.validate_csr(n, ncon, np.array(x), np.array(a),
                                      vwgt=None if vw is None else np.array(vw)) == 0
        try:
            rmb.Graph(n, ncon, x, a, vwgt=vw)
            got_ok = True
        except rmb.InputError:
            got_ok = False
        assert got_ok == want_ok, (x, a, vw)
