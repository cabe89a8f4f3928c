"""The identity behind the mixed form's grid-wide fast loop (no running sum of the barotropic wind per edge): with
dub_0 = 0 and dub_{j+1} = dub_j + tau (G - (Y_j[J] - Y_j[I]) / d_e), the sum over the n sub-steps of dub_j equals
tau (G n (n - 1) / 2 - (W[J] - W[I]) / d_e) with W = sum over j <= n - 2 of (n - 1 - j) Y_j per cell. Checked here in
FP64 on random edges and sub-step counts, with the cell-side accumulation in the order the cell pass keeps it (set at
sub-step 0, added to through sub-step n - 2)."""
import numpy as np
import pytest


@pytest.mark.parametrize('n', [1, 2, 7, 10, 20, 37])
def test_weighted_cell_sum_gives_the_sub_step_sum(n):
    rng = np.random.default_rng(n)
    E, N = 500, 300
    eI, eJ = rng.integers(0, N, E), rng.integers(0, N, E)
    G = rng.normal(size=E)
    rde = 1.0 / rng.uniform(5e4, 2e5, E)
    tau = 30.0
    Y = rng.normal(size=(n, N))
    dub = np.zeros(E)
    acc = np.zeros(E)
    W = np.zeros(N)
    for j in range(n):
        if j == 0:
            W = (n - 1) * Y[0]
        elif j <= n - 2:
            W = W + (n - 1 - j) * Y[j]
        acc += dub
        dub = dub + tau * (G - (Y[j][eJ] - Y[j][eI]) * rde)
    formed = tau * (G * (0.5 * n * (n - 1)) - (W[eJ] - W[eI]) * rde)
    scale = tau * n * (np.abs(G) + np.abs(Y).max() * rde) * n
    assert np.all(np.abs(formed - acc) <= 1e-12 * scale)
