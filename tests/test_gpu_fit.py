"""Calibration through the differentiable step (tests/material_fit_demo.py of the reference)."""

import numpy as np
import pytest
import torch

from newton_solver_diff_phd_b200.fit import CantileverFit, optimize
from newton_solver_diff_phd_b200.scenes import Cantilever

pytestmark = pytest.mark.gpu


def test_two_tetrahedron_material_fit_reduces_the_loss():
    result = optimize("cuda", iterations=15)
    # The reference demo's acceptance: at least 90 % of the trajectory loss removed.
    assert np.isfinite(result["final_loss"]) and result["final_loss"] < 0.1 * result["initial_loss"]


def test_batched_cantilever_fit_moves_young_toward_the_truth():
    rng = np.random.default_rng(4)
    specs = [Cantilever(nx, 2, 2, young, 0.4, rng.uniform(1.0, 5.0, 9))
             for nx, young in ((5, 3.0e5), (7, 1.0e6), (6, 6.0e5))]
    fit = CantileverFit(specs, steps=3, start_factor=2.0)
    optimizer = torch.optim.Adam([fit.log_young], lr=0.1)
    truth = np.log([spec.young for spec in specs])
    start_error = np.abs(fit.log_young.detach().cpu().numpy() - truth).max()
    losses = [fit.step(optimizer) for _ in range(6)]
    end_error = np.abs(fit.log_young.detach().cpu().numpy() - truth).max()
    assert losses[-1] < losses[0]
    assert end_error < 0.6 * start_error
