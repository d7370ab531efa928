"""Namelist reading: the oracle's reader against the reference examples, and
the library's own reader through the C-ABI (which reports parse errors
before it looks for a GPU)."""
import glob
import os

import pytest

from oracle.namelist import parse_namelist_text, read_namelist

HERE = os.path.dirname(os.path.abspath(__file__))
EXAMPLE = """&params
	! domain size
	nx_global = 34
	ny_global = 130
	nz_global = 34
	CFL = -0.001
	nu = 3.076923076923077e-04
	dPdx = 0.003275394114261
	x_mass_cte = 1 ! (0->use dPdx, 1->constant mass flow)
	filein = 'channel180_minchan.9999000'
	init_type = 0 ! (0->reads previous file, 1->zero, 2->random)
	grid_type = 1 ! (0->uniform, 1->stretched)
	body_type = 'none'
/
"""


def test_oracle_reader_values_and_defaults():
    p = parse_namelist_text(EXAMPLE)
    assert p["nx_global"] == 34 and p["ny_global"] == 130 and p["nz_global"] == 34
    assert p["cfl"] == -0.001 and p["nu"] == 3.076923076923077e-04
    assert p["filein"] == "channel180_minchan.9999000" and p["body_type"] == "none"
    assert p["alpha_stretch"] == 2.6 and p["cg_max_iter"] == 50   # defaults
    assert p["exterior_pressure_gradient"] is True


def test_oracle_reader_rejects_unknown():
    with pytest.raises(ValueError):
        parse_namelist_text("&params\n nx_global = 34\n bogus = 1\n/\n")


@pytest.mark.parametrize("text,msg", [
    ("&params\n nx_global = 34\n bogus = 1\n/\n", "unknown namelist variable"),
    ("&params\n nx_global = 3x4\n/\n", "bad integer"),
    ("&params\n nu = abc\n/\n", "bad real"),
    ("nx_global = 34\n", "no &params"),
])
def test_library_reader_errors(text, msg):
    import channel3d_parallel_b200 as c3d
    with pytest.raises(c3d.C3DError) as e:
        c3d.Channel(text=text)
    assert e.value.code == -1 and msg in str(e.value)


@pytest.mark.parametrize("nx,nz,which", [(35, 34, "nx"), (34, 29, "nz")])
def test_library_rejects_odd_nx_nz(nx, nz, which):
    import channel3d_parallel_b200 as c3d
    from channel3d_parallel_b200.channel import namelist_text
    with pytest.raises(c3d.C3DError) as e:
        c3d.Channel(text=namelist_text(nx_global=nx, ny_global=17, nz_global=nz, nu=1e-3, CFL=-1e-3))
    assert e.value.code == -1 and f"{which} must be even" in str(e.value)


def test_namelist_writer_roundtrip():
    from channel3d_parallel_b200.channel import namelist_text
    t = namelist_text(nx_global=194, ny_global=129, nz_global=194, nu=1 / 5600, CFL=-1e-3,
                      Lxp=12.566370614359172, body_type="none", exterior_pressure_gradient=False)
    p = parse_namelist_text(t)
    assert p["nu"] == 1 / 5600 and p["lxp"] == 12.566370614359172
    assert p["exterior_pressure_gradient"] is False
