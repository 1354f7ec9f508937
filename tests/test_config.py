"""LB3D namelist input: reader, defaults and derived values
(code/lb3d_config.F90)."""
import os

import pytest

from lb3d_b200.config import Params, parse_namelists, read_input
from tests._fixtures import GOLDEN


def test_quoted_slash_and_comments():
    g = parse_namelists("""
&variable_input
folder = './output/x'  ! a comment with / slash
beta = 10.000000, fr = 0.7
sci_od = .true.
/
""")
    v = g["variable_input"]
    assert v["folder"] == "./output/x"
    assert v["beta"] == 10.0 and v["fr"] == 0.7 and v["sci_od"] is True


def test_differential_file_overrides():
    p = read_input(os.path.join(GOLDEN, "gyroid", "gyroid.in"),
                   os.path.join(GOLDEN, "gyroid", "dump_xdr.din"))
    assert p.dump_format == "xdr"
    assert p.beta == 10.0 and p.g_ss == -0.003 and p.bdist == 2
    assert p.restore == 1 and p.init_cond == 7


def test_defaults_and_derived():
    p = read_input(os.path.join(GOLDEN, "wettingWall", "wettingWall.in"), ncomp=2)
    # rock_colour = 1.0 -> rock_colour_r (code/lb3d_config.F90:661-664)
    assert p.rock_colour_r == 1.0 and p.rock_colour_b == 0.0
    # g_accn_max* default to the lattice size (code/lb3d_config.F90:931-933)
    assert (p.g_accn_max, p.g_accn_max_x, p.g_accn_max_y) == (16, 16, 16)
    assert p.has_rock_file and p.obs_file == "wettingWall.wall.xdr"
    assert Params().tau_d == 2.0 and Params().beta == 1.0


def test_lees_edwards_flag_and_validation():
    p = read_input(os.path.join(GOLDEN, "leesEdwards", "leesEdwards.in"), ncomp=2)
    assert p.lees_edwards and p.shear_u == 0.01
    p.validate()
    p.ncomp = 3
    with pytest.raises(ValueError, match="Lees Edwards"):
        p.validate()


def test_sphere_pack_porosity_and_determinism():
    from lb3d_b200.ic import sphere_pack
    a = sphere_pack(48, 40, 32, seed=3, porosity=0.4, rmin=4, rmax=7, overlap=True)
    b = sphere_pack(48, 40, 32, seed=3, porosity=0.4, rmin=4, rmax=7, overlap=True)
    assert (a == b).all()
    assert abs(1.0 - a.mean() - 0.4) < 0.02
    c = sphere_pack(48, 40, 32, seed=3, porosity=0.4, rmin=4, rmax=7, overlap=False, max_tries=3000)
    assert 1.0 - c.mean() > 0.55  # non-overlapping spheres jam well before


def test_inflow_parameters_reach_the_c_struct():
    """fr, fg, fb and pr, pg, pb (code/lb3d_config.F90:169) and inv_type are
    read from the namelists with the reference's defaults and travel in
    lb3dc_params in the order include/lb3dc.h declares."""
    from lb3d_b200.config import params_from_namelists, to_cparams
    d = Params()
    assert (d.fr, d.fg, d.fb) == (1.0, 0.1, 0.5)
    g = parse_namelists("""
&fixed_input
nx = 8, ny = 8, nz = 6
/
&variable_input
boundary_cond = -1, inv_fluid = 11, inv_type = 1, bdist = 2
fr = 0.75, fb = 0.62, pr = 0.66, pb = 0.71, pg = 0.05
/
""")
    p = params_from_namelists(g, ncomp=2).finalize()
    p.validate()
    c = to_cparams(p)
    assert (c.inv_fluid, c.inv_type) == (11, 1)
    assert (c.fr, c.fb, c.pr, c.pb, c.pg, c.fg) == (0.75, 0.62, 0.66, 0.71, 0.05, 0.1)
    names = [n for n, _ in type(c)._fields_]
    assert names.index("fr") == names.index("pb") + 1 and names.index("precision") == names.index("fb") + 1
