"""Golden snapshot fixtures pinned to the reference's own reader.

Writes small snapshots with the oracle's restatement of output_data
(oracle/snapshot.py; src/input_output.f90:498-728) and decodes each with the
reference's Python reader ``read_field`` (tools/file_io.py:6-80 of the
reference tree), saving every record it returns.  The tests then check that
(1) the oracle writer still produces these exact bytes, (2) the library's
c3d_write_snapshot produces them too (GPU), and (3) the values the
reference's reader decoded are the state that was written.

Run from the repository root, in a container that has the reference tree:
    python tests/golden/make_snapshot_golden.py [path/to/reference]
"""
import importlib.util
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import channel_oracle as co      # noqa: E402
from oracle import ib_oracle as ibo          # noqa: E402
from oracle import snapshot as sn            # noqa: E402

NU = 1.0 / 5600.0


def plain_case():
    """12 x 9 x 8 channel (10 x 8 x 6 cells), seeded state, one RK3 step."""
    p = co.channel_params(12, 9, 8, 1.0, 0.7, NU, grid_type=1)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    co.compute_time_step_RK3(g, st, 1e-3)
    return p, g, st, None, None, None


def ib_case():
    """center_wall (src/immersed_boundary_geometry.f90:80-115) on a 10 x 17 x 10
    uniform grid, 8 x 8 markers, seeded marker unknowns fb, oracle Heaviside."""
    p = co.channel_params(10, 17, 10, 1.0, 0.5, NU, grid_type=0, alpha=0.0,
                          body_type="center_wall", nxb=8, nzb=8, cfl=-1e-3)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    ib = ibo.IBState(g, p, t=0.0)
    ibo.compute_heaviside(g, ib)
    fb = np.random.default_rng(3).standard_normal(4 * ib.body.nb)
    st.t = 0.125
    return p, g, st, ib.body, fb, (ib.Hu, ib.Hv, ib.Hw)


CASES = {
    "plain": (plain_case, False),
    "plain_original": (plain_case, True),
    "center_wall": (ib_case, False),
}


def case_bytes(name):
    make, original = CASES[name]
    p, g, st, body, fb, H = make()
    return sn.snapshot_bytes(g, st, 1e-3, body=body, fb=fb, H=H, original_format=original)


def main(ref_root):
    spec = importlib.util.spec_from_file_location("ref_file_io", os.path.join(ref_root, "tools", "file_io.py"))
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    for name, (make, original) in CASES.items():
        path = os.path.join(HERE, f"snapshot_{name}.bin")
        with open(path, "wb") as f:
            f.write(case_bytes(name))
        d = ref.read_field(path, original_format=original)
        np.savez(os.path.join(HERE, f"snapshot_{name}_ref_read.npz"),
                 **{k: np.asarray(v) for k, v in d.items()})
        print(name, os.path.getsize(path), "bytes,", len(d), "records")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
