"""Binary state file, CPU side: round trip, corruption detection, and exact resume of the CPU
restatement (and of the reference's own code when its build is present) from a file."""
import numpy as np
import pytest

import oracle
from oracle import Oracle2D
from oracle.state_format import read_state, write_state

QUAD = dict(num_levels=4, nx_coarse=9, ny_coarse=9, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0)
GEOM = (4, 9, 9, 0, 0.0, 1.0, 0.0, 1.0, 1.4)


def stepped(kind, n, tol=1e-3, cfl=0.4):
    o = Oracle2D(**QUAD, bc_kind=0, kind=kind)
    o.init_problem(0, 0.5, 0.5)
    t = 0.0
    for _ in range(n):
        t += o.step(tol, cfl, t, 10.0)[0]
    return o, t


def test_round_trip(tmp_path):
    o, t = stepped("port", 3)
    q, m, lv = o.get_q(), o.get_masks(), o.get_levels()
    p = tmp_path / "s.bin"
    write_state(p, GEOM, q, m, lv, t, 3)
    r = read_state(p)
    assert r["t"] == t and r["step"] == 3 and r["geometry"] == GEOM
    assert np.array_equal(r["masks"], m) and np.array_equal(r["levels"], lv)
    on = m[1, 3:-3, 3:-3].astype(bool)
    assert np.array_equal(r["q"][3:-3, 3:-3][on], q[3:-3, 3:-3][on])
    # between steps everything off mask0 is zero in the interior (PostProcessEuler)
    assert np.all(q[4:-4, 4:-4][~on[1:-1, 1:-1]] == 0)


def test_corruption_detected(tmp_path):
    o, t = stepped("port", 1)
    p = tmp_path / "s.bin"
    write_state(p, GEOM, o.get_q(), o.get_masks(), o.get_levels(), t, 1)
    raw = bytearray(p.read_bytes())
    raw[200] ^= 0x01
    bad = tmp_path / "bad.bin"
    bad.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="CRC"):
        read_state(bad)
    raw = bytearray(p.read_bytes())
    raw[0:8] = b"XXXXXXXX"
    bad.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="not an AWCM"):
        read_state(bad)
    bad.write_bytes(p.read_bytes()[:-8])
    with pytest.raises(ValueError, match="size"):
        read_state(bad)


@pytest.mark.parametrize("kind", ["port", "reference"])
def test_resume_from_file_is_exact(tmp_path, kind):
    if kind == "reference" and not oracle.reference_available():
        pytest.skip("reference build absent")
    full, t_full = stepped(kind, 6)
    part, t = stepped(kind, 3)
    p = tmp_path / "s.bin"
    write_state(p, GEOM, part.get_q(), part.get_masks(), part.get_levels(), t, 3)
    r = read_state(p)
    o = Oracle2D(**QUAD, bc_kind=0, kind=kind)
    o.set_q(r["q"])
    o.set_masks(r["masks"])
    o.set_levels(r["levels"])
    t = r["t"]
    for _ in range(3):
        t += o.step(1e-3, 0.4, t, 10.0)[0]
    assert t == t_full
    assert np.array_equal(o.get_q()[3:-3, 3:-3], full.get_q()[3:-3, 3:-3])
    assert np.array_equal(o.get_masks(), full.get_masks())
