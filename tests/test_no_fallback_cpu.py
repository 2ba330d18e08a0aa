"""Without a GPU every compute entry point fails with XG_ERR_CUDA: the
library has no CPU fallback (runs only where torch sees no CUDA device)."""
import numpy as np
import pytest


def _no_gpu():
    try:
        import torch

        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_compute_entry_points_fail_without_a_gpu(xg):
    x, y = xg.generate_xy_loc(100, 0)
    z = np.ones(100)
    calls = [
        lambda: xg.dmle_host(x, y, z, [1.0, 0.1, 0.5]),
        lambda: xg.dmle_host_sliced(x, y, z, [1.0, 0.1, 0.5]),
        lambda: xg.dmle_host_mixed(x, y, z, [1.0, 0.1, 0.5], ts=256),
        lambda: xg.fisher_host(x, y, [1.0, 0.1, 0.5]),
        lambda: xg.mloe_mmom_host(x[:10], y[:10], x[10:], y[10:], [1.0, 0.1, 0.5], [1.0, 0.1, 0.5]),
        lambda: xg.covariance_dense(x, y, [1.0, 0.1, 0.5]),
        lambda: xg.dmle_host(x, y, np.ones(200), [1.0, 1.0, 0.1, 0.5, 0.5, 0.3], kernel=2),
    ]
    for call in calls:
        with pytest.raises(xg.XgError) as ei:
            call()
        assert ei.value.code == xg.XG_ERR_CUDA
