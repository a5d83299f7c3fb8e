"""Namelist input of the run loop (sph_read_namelist), on the host: the
reference's &grid and &boxparams groups (grid_init, box_init,
src/pseudo/pseudospec_mod.f90:41-69,151-160) and the loop's &run group."""
import pytest

from redondito_b200 import sphp as S

GOOD = """! a run at the first benchmark configuration
&grid
  lmax = 31, nz = 58,
  Cz = 25, oz = 5   ! continuation points, matching order
/
&BOXPARAMS rint=0.35D0, rext=1.0d0 /
&run dt=1.0D-4 step=10 tstep=2 sstep=5 nu=1e-3 filter=.true. /
"""


def test_namelist_groups_and_formats(tmp_path):
    f = tmp_path / "run.nml"
    f.write_text(GOOD)
    d = S.read_namelist(str(f))
    assert (d["lmax"], d["nz"], d["Cz"], d["oz"]) == (31, 58, 25, 5)
    assert (d["rint"], d["rext"]) == (0.35, 1.0)
    assert (d["dt"], d["step"], d["tstep"], d["sstep"], d["nu"], d["filter"]) == (1e-4, 10, 2, 5, 1e-3, True)


def test_namelist_defaults(tmp_path):
    """grid_init sets Cz = oz = 0 when the namelist leaves them out; the run
    group is optional."""
    f = tmp_path / "run.nml"
    f.write_text("&grid lmax=7, nz=16 /\n&boxparams rint=0.5, rext=1.5 /\n")
    d = S.read_namelist(str(f))
    assert (d["lmax"], d["nz"], d["Cz"], d["oz"]) == (7, 16, 0, 0)
    assert (d["dt"], d["step"], d["tstep"], d["sstep"], d["nu"], d["filter"]) == (0.0, 0, 1, 0, 0.0, False)


@pytest.mark.parametrize("text", [
    "&grid lmax=7 /\n",                                                  # no boxparams
    "&grid lmax=7, nz=16 /\n&boxparams rint=0.5 /\n",                     # rext missing
    "&grid lmax=7, nz=16, nlat=12 /\n&boxparams rint=0.5, rext=1.5 /\n",  # unknown key
    "&grid lmax=7.5, nz=16 /\n&boxparams rint=0.5, rext=1.5 /\n",         # not an integer
    "&grid lmax=7, nz=16 /\n&boxparams rint=x, rext=1.5 /\n",             # not a number
    "&grid lmax=7, nz=16\n&boxparams rint=0.5, rext=1.5\n",               # no terminator
])
def test_namelist_errors(tmp_path, text):
    f = tmp_path / "bad.nml"
    f.write_text(text)
    with pytest.raises(S.SphError) as e:
        S.read_namelist(str(f))
    assert e.value.code == 1


def test_namelist_missing_file(tmp_path):
    with pytest.raises(S.SphError) as e:
        S.read_namelist(str(tmp_path / "none.nml"))
    assert e.value.code == 5
