"""The learned sparse-transmit path with the committed trained weights, on held-out phantoms.

Shows what the trained network gains over the method without it: the NRMSE of the restored
volume against the plain full-transmit volume, next to the NRMSE of the sparse delay-and-sum
volume itself, on phantoms the network never saw (seeds from 1 000 000). Also checks that the
gate's spot-check estimate tracks the true NRMSE and that rejected volumes are charged a
fallback.
"""
import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200 import sparse

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def evaluation():
    net = sparse.load()
    summary, rows = sparse.evaluate(net, 4, warmup=1)
    net.close()
    return summary, rows


def test_network_improves_on_sparse_das(evaluation):
    _, rows = evaluation
    for r in rows:
        # measured on 256 held-out phantoms: median 0.38 restored vs 0.78 sparse
        assert r["nrmse_net"] < 0.6 * r["nrmse_plain"], r


def test_gate_estimate_tracks_true_nrmse(evaluation):
    _, rows = evaluation
    for r in rows:
        # a 1/64 tile sample: ~10 % median relative error over 256 held-out volumes
        assert abs(r["gate_nrmse"] - r["nrmse_net"]) < 0.3 * r["nrmse_net"] + 0.02, r


def test_rejected_volumes_are_charged_the_fallback(evaluation):
    summary, rows = evaluation
    n = len(rows)
    ok = [r["gate_nrmse"] <= sparse.NRMSE_BAR for r in rows]
    learned_ms = sum(r["sparse_ms"] + r["unet_ms"] + r["front_ms"] + r["gate_ms"] + (0 if g else r["das_ms"])
                     for r, g in zip(rows, ok))
    assert abs(summary["learned_volumes_per_s"] - 1e3 * n / learned_ms) < 1e-6 * summary["learned_volumes_per_s"]
    assert summary["gate_pass_fraction"] == sum(ok) / n
