"""The shot driver's file readers against the reference's own: the parameter
file (Inversion::readParamFile with ParserFromFile rules) and the coordinate
file (Coords).  Host-only."""

import numpy as np
import pytest

import oracle as O
from seis_b200 import driver

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference oracle not built")

BASE = """! survey written for the reader test
nthread   4
ns        {ns}
ngmax     {ngmax}      ! largest shot
nx        300
nz        120
nt        2000
{npml}
delay     10
delaycal  {delaycal}
mask      {mask}
maxiter   7
lpad {lpad}
rpad 25
sbegin 0
send   {send}
dx 0.010
dz {dz}
dt 0.0016
fr 25
{velfx}
planeTag  0
precsg     {d}/CSG/CSG
wdir       {d}/WDIR/
vfile      {d}/v.bin
v0file     {d}/v0.bin
coordfile  {d}/coords.txt
{maskfile}
"""


@pytest.mark.parametrize("variant", range(5))
def test_parameter_file_matches_reference(tmp_path, variant):
    kw = dict(ns=[3, 300, 12, 1, 50][variant], ngmax=[298, 5, 9, 1, 77][variant],
              npml=["npml 20", "", "npml   35 ! pad", "npml 7", ""][variant],
              delaycal=[500, 0, 94, 120, 75][variant], mask=[1, 0, 0, 1, 0][variant],
              lpad=[50, 0, 3, 10, 40][variant], send=[2, 299, 11, 0, 49][variant],
              dz=["0.010", "12.5", "1e-2", ".5", "+7.5"][variant],
              velfx=["velfx 0.0", "", "velfx -3.5", "velfx 12", ""][variant],
              maskfile=["maskfile {d}/mask.bin", "", "", "maskfile {d}/m.bin ! mute", ""][variant],
              d=str(tmp_path))
    kw["maskfile"] = kw["maskfile"].format(d=tmp_path)
    path = tmp_path / "param.txt"
    path.write_text(BASE.format(**kw))
    want = O.ref_read_params(str(path))
    got = driver.read_params(str(path)).as_dict()
    assert want is not None
    for k, v in want.items():
        if k == "maskfile" and not got["mask"]:
            continue  # not read by the reference unless mask = 1
        assert got[k] == v, (k, got[k], v)


def test_parameter_file_missing_required_key(tmp_path):
    path = tmp_path / "param.txt"
    path.write_text("ns 3\nngmax 4\nnx 10\n")
    with pytest.raises(Exception):
        driver.read_params(str(path))


def write_coords(path, shots, trailing_newline=True):
    lines = []
    for (sx, sz), recs in shots:
        for gx, gz in recs:
            lines.append(f"{sx:.4f} {sz:.4f} {gx:.4f} {gz:.4f}")
    text = "\n".join(lines) + ("\n" if trailing_newline else "")
    path.write_text(text)


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("trailing", [True, False])
def test_coordinate_file_matches_reference(tmp_path, seed, trailing):
    rng = np.random.default_rng(seed)
    shots = []
    for i in range(int(rng.integers(1, 7))):
        sx = 100.0 + 37.5 * i
        ng = int(rng.integers(1, 40))
        recs = [(float(rng.uniform(0, 3000)), float(rng.integers(0, 4) * 12.5)) for _ in range(ng)]
        shots.append(((sx, float(rng.integers(0, 3) * 10.0)), recs))
    path = tmp_path / "coords.txt"
    write_coords(path, shots, trailing)
    ngmax = max(len(r) for _, r in shots) + 1
    ns, ng_ref, sc_ref, gc_ref = O.ref_read_coords(str(path), ngmax)
    ng, sc, gc = driver.read_coords(str(path), ngmax)
    assert len(ng) == ns
    assert np.array_equal(ng, ng_ref)
    assert np.array_equal(sc, sc_ref)
    for i in range(ns):  # the receivers each shot counts
        assert np.array_equal(gc[i, :, :ng[i]], gc_ref[i, :, :ng_ref[i]])
    if trailing:
        assert list(ng) == [len(r) for _, r in shots]
