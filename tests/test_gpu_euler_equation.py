"""EULER_EQUATION_1D/2D batch entry points on the GPU (euler1d_flux, euler1d_spectral_radius,
euler2d_flux, euler2d_spectral_radius) against the reference's own EULER_EQUATION classes and the
CPU restatement, bit for bit, on seeded gas states (density and pressure log-uniform over four
decades, velocities of both signs), an empty batch included."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def gas_states(n, dim, seed):
    rng = np.random.default_rng(seed)
    rho = 10.0 ** rng.uniform(-2, 2, n)
    p = 10.0 ** rng.uniform(-2, 2, n)
    vel = rng.uniform(-3, 3, (n, dim))
    E = p / 0.4 + 0.5 * rho * (vel ** 2).sum(axis=1)
    return np.column_stack([rho, rho[:, None] * vel, E])


def kinds():
    return ["port", "reference"] if oracle.reference_available() else ["port"]


@pytest.mark.parametrize("dim,direction", [(1, 0), (2, 0), (2, 1)])
@pytest.mark.parametrize("n", [0, 1, 1000, 65537])
def test_flux_and_spectral_radius(awcm_lib, dim, direction, n):
    import torch

    q = gas_states(n, dim, 11 + n + dim + direction)
    qd = torch.tensor(q, dtype=torch.float64, device="cuda").contiguous()
    fd = torch.full_like(qd, np.nan)
    sd = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
    awcm_lib.euler_flux(qd.data_ptr(), fd.data_ptr(), n, dim, direction)
    awcm_lib.euler_spectral_radius(qd.data_ptr(), sd.data_ptr(), n, dim, direction)
    torch.cuda.synchronize()
    f, s = fd.cpu().numpy(), sd.cpu().numpy()
    for kind in kinds():
        assert np.array_equal(f, oracle.euler_flux(q, dim, direction, kind=kind)), kind
        assert np.array_equal(s, oracle.euler_spectral_radius(q, dim, direction, kind=kind)), kind


def test_bad_arguments(awcm_lib):
    with pytest.raises(awcm_lib.AwcmError):
        awcm_lib.euler_flux(0, 0, 5, 2, 2)
    with pytest.raises(awcm_lib.AwcmError):
        awcm_lib.euler_flux(0, 0, -1, 1)
