"""Host logic of the surrogate-screened calibration (CPU): the interface's rates, the frame
features, the fitness and the error measures."""

import numpy as np
import torch

from flyzero_b200 import tuning as T


def test_interface_rates_follow_the_parameters():
    rng = np.random.default_rng(0)
    xy = torch.as_tensor(rng.random((400, 2)).astype(np.float32))
    x = torch.as_tensor(rng.random((5, T.N_PARAMS)).astype(np.float32))
    r = T.interface_rates(x, xy, 33.0)
    p = T.unit_to_params(x)
    assert r.shape == (5, 401)
    assert torch.all(r[:, :400] >= 0) and torch.all(r[:, :400] <= p[:, 8:9] + 1e-4)      # rate cap
    assert torch.allclose(r[:, 400], p[:, 9])                                              # tonic drive
    hidden = xy[:, 1][None, :] < p[:, 1:2]                                                  # above y_min
    assert torch.all(r[:, :400][hidden] == 0)


def test_features_bin_expected_input_counts_by_patch():
    rng = np.random.default_rng(1)
    xy = rng.random((3000, 2)).astype(np.float32)
    f = T.Featurizer(xy, torch.device("cpu"))
    rates = torch.as_tensor(rng.uniform(0, 200, (2, 3001)).astype(np.float32))
    prev = torch.as_tensor(rng.poisson(2.0, (2, 10)).astype(np.float32))
    X = f(rates, prev)
    cell = np.minimum((xy * 32).astype(int), 31)
    patch = cell[:, 1] * 32 + cell[:, 0]
    want = np.zeros((2, 1024))
    np.add.at(want.T, patch, (rates[:, :3000].numpy() * (T.wl.FRAME_MS / 1000.0)).T)
    np.testing.assert_allclose(X[:, :1024].numpy(), np.log1p(want), atol=1e-5)
    np.testing.assert_allclose(X[:, 1024:].numpy(), np.log1p(prev.numpy()) @ f.P.numpy().T, rtol=1e-5, atol=1e-5)


def test_fitness_and_errors():
    c = np.zeros((2, 3, 10))
    c[0, :, 8] = 2.0                  # forward only
    c[1, :, 0] = 4.0                  # one-sided steering
    f = T.fitness(c)
    assert f[0] == 2.0 and f[1] == 0.25 * 4 - 0.5 * 4
    assert T.count_error(c, c).max() == 0 and T.aggregate_count_error(c * 1.1, c) > 0.099
