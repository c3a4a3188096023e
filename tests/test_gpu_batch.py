"""GPU: homogeneous collision steps for a batch of instances of different grid
sizes (one batched launch sequence per size) against the oracle's
CollisionStep / RK4 per instance."""
import numpy as np
import pytest

import orc
import qbgpu
from conftest import rel_l1

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

J, M, L, R = 4, 3, 6.0, 3.75
TOL = 1e-12


@pytest.mark.parametrize("rk4", [True, False])
def test_mixed_size_batch_matches_oracle(rk4):
    sizes = [8, 16, 8, 32, 16, 8]
    rng = np.random.default_rng(11)
    Wf = [orc.to_fourier(qbgpu.gaussian_mixture_state(n, L, seed=100 + i, ncells=1))[0] for i, n in enumerate(sizes)]
    B = rng.standard_normal((len(sizes), 3)) * 0.1
    states = [torch.from_numpy(w.copy()).cuda() for w in Wf]
    dt, steps = 0.01, 2
    qbgpu.homogeneous_batch(states, dt, steps, B=B, rk4=rk4, J=J, M=M, L=L, R=R)
    oracles = {n: orc.Oracle(n, J, M, L, R) for n in set(sizes)}
    for i, n in enumerate(sizes):
        ref = Wf[i]
        for _ in range(steps):
            ref = oracles[n].collision_step(ref, dt, B[i], rk4=rk4)
        assert rel_l1(states[i].cpu().numpy(), ref) < TOL, (i, n)


def test_batch_rejects_unsupported_size():
    bad = [torch.zeros((4, 24, 24), dtype=torch.complex128, device="cuda")]
    with pytest.raises(RuntimeError, match="N=24"):
        qbgpu.homogeneous_batch(bad, 0.01, 1, J=J, M=M, L=L, R=R)
