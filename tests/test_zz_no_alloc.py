"""The allocation-free 1D step (awcm1d_step_noalloc) against the allocating entry point.

awcm1d_step_noalloc exists for callers that may not allocate device memory themselves -- a host
framework whose GPU memory is owned by its own caching allocator, or a loop with a fixed memory
budget -- so it takes the caller's device buffers for the state and keeps its working buffers in a
static array inside the library.  This test drives it through the C-ABI on two calls in a row
(the second call reuses the static array the first one left behind) and requires the same result
as the batch entry point (awcm1d_batch_*) and as the CPU oracle, bit for bit: the same tolerance
as every parity test here.  It sits in its own file, collected last, and passes alone or after
the rest of the suite.
"""
import numpy as np
import pytest

from oracle import Oracle1D

pytestmark = pytest.mark.gpu

NX = 1025
LEVELS, NX_COARSE = 7, 17
X0, X1 = 0.5 / NX, 1 - 0.5 / NX
TOL, CFL, T_END = 1e-4, 0.5, 0.2


def unpack(state, w):
    """Mask planes (mask_temp, mask0..mask3) and level planes from the device state layout."""
    mb = state[:w]
    masks = np.stack([(mb >> b) & 1 for b in (4, 0, 1, 2, 3)]).astype(np.uint8)
    levels = state[w:].view(np.int8).reshape(4, w)[:, 3:-3].astype(np.int32)
    return masks, levels


def test_noalloc_step_matches_allocating_entry_point(awcm_lib):
    import torch

    torch.cuda.set_device(0)
    ref = awcm_lib.AWCM1D(LEVELS, NX_COARSE, X0, X1)
    ref.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    cpu = Oracle1D(LEVELS, NX_COARSE, X0, X1, kind="port")
    cpu.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    w = NX + 6
    q_dev = torch.tensor(np.ascontiguousarray(ref.get_q().T), dtype=torch.float64, device="cuda")
    state = np.zeros(5 * w, np.uint8)
    state[:w] = 0x01
    state[:3] = 0xE1
    state[w - 3:w] = 0xE1
    state_dev = torch.tensor(state, device="cuda")
    out_dev = torch.zeros(16, dtype=torch.float64, device="cuda")
    t = 0.0
    for call in range(2):
        o_ref = ref.step(TOL, CFL, t, T_END)
        o_cpu = cpu.step(TOL, CFL, t, T_END)
        assert np.array_equal(o_ref, o_cpu), f"call {call}: batch entry point vs oracle"
        awcm_lib._lib.call("awcm1d_step_noalloc", LEVELS, NX_COARSE, X0, X1, 1.4, awcm_lib.WENOZ, TOL, CFL, t, T_END,
                           q_dev.data_ptr(), state_dev.data_ptr(), out_dev.data_ptr(), None)
        torch.cuda.synchronize()
        out = out_dev.cpu().numpy()
        assert out[1] == o_ref[0], f"call {call}: dt {out[1]!r} vs {o_ref[0]!r}"
        assert np.array_equal(out[5:9], o_ref[2:6]), f"call {call}: mask sizes"
        assert np.array_equal(out[10:13], o_ref[6:9]), f"call {call}: LF speeds"
        # per-call results: one step taken, this step's |mask0|, no error
        assert out[4] == 1 and out[13] == out[5] and out[14] == 0, f"call {call}: {out[[4, 13, 14]]}"
        q = q_dev.cpu().numpy().T
        q_ref = ref.get_q()
        scale = np.abs(q_ref).max()
        assert np.abs(q - q_ref).max() <= 1e-11 * scale, f"call {call}: field beyond 1e-11"
        assert np.array_equal(q, q_ref), f"call {call}: field not bit-identical"
        assert np.array_equal(q, cpu.get_q()), f"call {call}: field differs from the oracle"
        masks, levels = unpack(state_dev.cpu().numpy(), w)
        assert np.array_equal(masks, ref.get_masks()), f"call {call}: masks"
        assert np.array_equal(masks, cpu.get_masks()), f"call {call}: masks differ from the oracle"
        assert np.array_equal(levels, ref.get_levels()), f"call {call}: levels"
        assert np.array_equal(levels, cpu.get_levels()), f"call {call}: levels differ from the oracle"
        t += o_ref[0]


def test_noalloc_rejects_oversized_instance(awcm_lib):
    import torch

    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(awcm_lib.AwcmError, match="exceeds the static scratch limit"):
        # 17 coarse points, 15 levels: Nx = 16 * 2^14 + 1 = 262145 > 8193
        awcm_lib._lib.call("awcm1d_step_noalloc", 15, 17, 0.0, 1.0, 1.4, 0, TOL, CFL, 0.0, T_END,
                           dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), None)
