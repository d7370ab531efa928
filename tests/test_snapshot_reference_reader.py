"""The snapshot format pinned to the reference's own reader.

``tests/golden/snapshot_*.bin`` were written by the oracle's output_data
restatement and decoded by the reference's ``read_field``
(tools/file_io.py:6-80) into ``snapshot_*_ref_read.npz``
(tests/golden/make_snapshot_golden.py).  Here: the oracle writer still makes
those bytes, and what the reference's reader decoded is the written state,
record by record.  Where the reference tree is present its reader is also run
live on the committed files.  The GPU side (c3d_write_snapshot producing the
same bytes) is in tests/test_gpu_io.py.
"""
import importlib.util
import os

import numpy as np
import pytest

from oracle import snapshot as sn

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
REF_READER = os.path.join("/root/reference", "tools", "file_io.py")


def _gen():
    spec = importlib.util.spec_from_file_location("make_snapshot_golden",
                                                  os.path.join(GOLD, "make_snapshot_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


GEN = _gen()
NAMES = list(GEN.CASES)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_writer_reproduces_golden_bytes(name):
    with open(os.path.join(GOLD, f"snapshot_{name}.bin"), "rb") as f:
        assert GEN.case_bytes(name) == f.read()


@pytest.mark.parametrize("name", NAMES)
def test_reference_reader_decoded_the_written_state(name):
    make, original = GEN.CASES[name]
    p, g, st, body, fb, H = make()
    ref = np.load(os.path.join(GOLD, f"snapshot_{name}_ref_read.npz"))
    want = {"x": g.x[1:], "y": g.y[1:], "z": g.z[1:],
            "xm": g.xm[1:g.nx], "ym": g.ym[1:g.ny], "zm": g.zm[1:g.nz],
            "U": st.U[1:, 1:, 1:], "V": st.V[1:, 1:, 1:], "W": st.W[1:, 1:, 1:],
            "P": st.P[1:, 1:, 1:]}
    # the reader rebuilds the ghost-centre grids the solver uses
    want.update(xg=g.xg[1:], yg=g.yg[1:], zg=g.zg[1:])
    if not original:
        Hs = H if H is not None else tuple(np.ones_like(a) for a in (st.U, st.V, st.W))
        want.update(Hu_interior=Hs[0][1:, 1:, 1:], Hv_interior=Hs[1][1:, 1:, 1:],
                    Hw_interior=Hs[2][1:, 1:, 1:], t=st.t, dt=1e-3, dpdx=st.dPdx, nu=p["nu"],
                    nxb=p["nxb"], nzb=p["nzb"])
        if body is not None:
            want.update(xb=body.xb, yb=body.yb, zb=body.zb, fb=fb, ub=body.ub, sb=body.sb,
                        normals=body.normals, tangents_1=body.tangents_1,
                        tangents_2=body.tangents_2)
        else:
            for k in ("xb", "yb", "zb", "fb", "ub", "sb", "normals", "tangents_1", "tangents_2"):
                want[k] = np.zeros(0)
    assert set(ref.files) == set(want), sorted(set(ref.files) ^ set(want))
    for k, v in want.items():
        a = ref[k]
        if k in ("xg", "yg", "zg"):
            # computed by the reader from x and xm (tools/file_io.py:38-40)
            assert np.allclose(a, v, rtol=0, atol=1e-15), k
        else:
            assert np.array_equal(a, np.asarray(v)), k
    # and the oracle's own reader agrees with the reference's on every record
    d = sn.read_snapshot(os.path.join(GOLD, f"snapshot_{name}.bin"))
    for k in d:
        if k in ref.files:
            assert np.array_equal(np.asarray(d[k]), ref[k]), k


@pytest.mark.skipif(not os.path.exists(REF_READER), reason="reference tree not present")
@pytest.mark.parametrize("name", NAMES)
def test_reference_reader_live(name):
    spec = importlib.util.spec_from_file_location("ref_file_io", REF_READER)
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    _, original = GEN.CASES[name]
    d = ref.read_field(os.path.join(GOLD, f"snapshot_{name}.bin"), original_format=original)
    stored = np.load(os.path.join(GOLD, f"snapshot_{name}_ref_read.npz"))
    assert set(d) == set(stored.files)
    for k, v in d.items():
        assert np.array_equal(np.asarray(v), stored[k]), k
