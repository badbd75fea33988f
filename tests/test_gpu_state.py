"""Binary state file on the GPU: the product's files read by the checker, the checker's files
loaded by the product, exact resume, and rejection of damaged or mismatched files."""
import numpy as np
import pytest

from oracle import Oracle2D
from oracle.state_format import read_state, write_state

pytestmark = pytest.mark.gpu

QUAD = (4, 9, 9, 0.0, 1.0, 0.0, 1.0)
DMACH = (4, 17, 5, 0.0, 4.0, 0.0, 1.0)


def gpu_stepped(awcm, n, geom=QUAD, bc=0, prob=0, a=0.5, b=0.5, tol=1e-3, cfl=0.4):
    s = awcm.AWCM2D(*geom, bc_kind=bc)
    s.init_problem(prob, a, b)
    t = 0.0
    for _ in range(n):
        t += s.step(tol, cfl, t, 10.0)[0]
    return s, t


def test_product_file_read_by_checker(tmp_path, awcm_lib):
    s, t = gpu_stepped(awcm_lib, 3)
    p = tmp_path / "g.bin"
    s.save_state(p, t, 3)
    r = read_state(p)
    assert r["t"] == t and r["step"] == 3
    assert r["geometry"] == s.geometry()
    assert np.array_equal(r["masks"], s.get_masks())
    assert np.array_equal(r["levels"], s.get_levels())
    on = r["masks"][1, 3:-3, 3:-3].astype(bool)
    assert np.array_equal(r["q"][3:-3, 3:-3][on], s.get_q()[3:-3, 3:-3][on])


def test_checker_file_loaded_by_product(tmp_path, awcm_lib):
    """A state written by the checker after 3 steps of its own, loaded on the GPU, then 3 more
    steps on both sides: identical."""
    o = Oracle2D(*QUAD, bc_kind=0, kind="port")
    o.init_problem(0, 0.5, 0.5)
    t = 0.0
    for _ in range(3):
        t += o.step(1e-3, 0.4, t, 10.0)[0]
    p = tmp_path / "o.bin"
    write_state(p, (4, 9, 9, 0, *QUAD[3:], 1.4), o.get_q(), o.get_masks(), o.get_levels(), t, 3)
    s = awcm_lib.AWCM2D(*QUAD, bc_kind=0)
    tg, step = s.load_state(p)
    assert tg == t and step == 3
    for _ in range(3):
        dr = o.step(1e-3, 0.4, t, 10.0)[0]
        dg = s.step(1e-3, 0.4, t, 10.0)[0]
        assert dg == dr
        t += dr
    assert np.array_equal(s.get_masks(), o.get_masks())
    assert np.array_equal(s.get_q()[3:-3, 3:-3], o.get_q()[3:-3, 3:-3])


@pytest.mark.parametrize("case", ["quad", "dmach"])
def test_resume_is_exact(tmp_path, awcm_lib, case):
    kw = dict(geom=QUAD) if case == "quad" else dict(geom=DMACH, bc=1, prob=1, a=1.4, b=0.0, cfl=0.5)
    full, t_full = gpu_stepped(awcm_lib, 8, **kw)
    part, t = gpu_stepped(awcm_lib, 4, **kw)
    p = tmp_path / "r.bin"
    part.save_state(p, t, 4)
    s = awcm_lib.AWCM2D(*kw["geom"], bc_kind=kw.get("bc", 0))
    t, step = s.load_state(p)
    for _ in range(4):
        t += s.step(1e-3, kw.get("cfl", 0.4), t, 10.0)[0]
    assert t == t_full
    assert np.array_equal(s.get_masks(), full.get_masks())
    assert np.array_equal(s.get_q()[3:-3, 3:-3], full.get_q()[3:-3, 3:-3])


def test_damaged_and_mismatched_files_rejected(tmp_path, awcm_lib):
    s, t = gpu_stepped(awcm_lib, 2)
    p = tmp_path / "g.bin"
    s.save_state(p, t, 2)
    q_before, m_before = s.get_q(), s.get_masks()
    raw = bytearray(p.read_bytes())
    raw[300] ^= 0x10
    bad = tmp_path / "bad.bin"
    bad.write_bytes(bytes(raw))
    with pytest.raises(awcm_lib.AwcmError, match="CRC"):
        s.load_state(bad)
    other = awcm_lib.AWCM2D(4, 9, 9, 0.0, 2.0, 0.0, 1.0, bc_kind=0)
    with pytest.raises(awcm_lib.AwcmError, match="geometry"):
        other.load_state(p)
    with pytest.raises(awcm_lib.AwcmError):
        s.load_state(tmp_path / "missing.bin")
    short = tmp_path / "short.bin"
    short.write_bytes(p.read_bytes()[:-16])
    with pytest.raises(awcm_lib.AwcmError, match="truncated payload"):
        s.load_state(short)
    short.write_bytes(p.read_bytes()[:100])
    with pytest.raises(awcm_lib.AwcmError, match="truncated header"):
        s.load_state(short)
    # a state of another gas (gamma 1.3) is refused: its energies mean other pressures
    r = read_state(p)
    g13 = tmp_path / "g13.bin"
    write_state(g13, r["geometry"][:-1] + (1.3,), r["q"], r["masks"], r["levels"], r["t"], r["step"])
    with pytest.raises(awcm_lib.AwcmError, match="gamma") as ei:
        s.load_state(g13)
    assert ei.value.status == 6
    # every rejection above left the instance as it was
    assert np.array_equal(s.get_q(), q_before) and np.array_equal(s.get_masks(), m_before)
