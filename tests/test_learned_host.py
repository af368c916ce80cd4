"""Host-side pieces of the learned preconditioner and of recursive
checkpointing that need no GPU: feature normalisation, random training
models, the two-level segment choice, the U-Net parameter layout."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_features_normalise_and_pad():
    from seispie_b200.learned import features
    nx, nz = 20, 13
    rng = np.random.default_rng(0)
    g = torch.as_tensor(rng.standard_normal(nx * nz), dtype=torch.float32)
    illum = torch.as_tensor(rng.random(nx * nz) ** 4 * 1e6, dtype=torch.float32)
    m = torch.as_tensor(1e10 * (1 + 0.1 * rng.standard_normal(nx * nz)), dtype=torch.float32)
    f = features(g, illum, m, nx, nz)
    assert f.shape == (1, 3, 24, 16)
    assert float(f[0, 0].abs().max()) == pytest.approx(1.0)
    assert float(f[0, 1, :nx, :nz].min()) >= 0.0
    assert float(f[0, 1].max()) == pytest.approx(1.0, abs=1e-4)
    assert abs(float(f[0, 2, :nx, :nz].mean())) < 1e-5
    assert torch.all(f[0, :, nx:, :] == 0) and torch.all(f[0, :, :, nz:] == 0)


def test_random_boards_are_bounded():
    from seispie_b200.learned import random_board
    rng = np.random.default_rng(1)
    for _ in range(20):
        b = random_board(rng, 64, 48)
        assert b.shape == (64, 48) and np.abs(b).max() <= 1.0 + 1e-12 and np.abs(b).max() > 0.5


def test_two_level_segments_minimise_memory():
    from seispie_b200._lib import FWI_PSV, FWI_SPIN
    from seispie_b200.adjoint import two_level_segments
    from seispie_b200.engine import NS, NV
    from seispie_b200.adjoint import strain_fields
    for mode, nt in ((FWI_SPIN, 8000), (FWI_PSV, 4000), (FWI_PSV, 7)):
        k1, k2 = two_level_segments(nt, mode)
        assert 1 <= k2 <= k1 <= nt
        S, P = NS[mode] + 2 * NV[mode], strain_fields(mode) + NV[mode]

        def mem(a, b):
            return S * (math.ceil(nt / a) + math.ceil(a / b)) + P * b
        best = min(mem(a, b) for a in range(1, min(nt, 2000) + 1, 7) for b in range(1, min(a, 200) + 1, 3))
        assert mem(k1, k2) <= 1.1 * best


def test_unet_layout_is_aligned_and_complete():
    from seispie_b200.unet import LAYERS
    # the flat layout of UNet.__init__, without touching a device
    off, seen = 0, []
    for name, c0, c1, co in LAYERS:
        assert c0 % 16 == 0 and c1 % 16 == 0 and co % 16 == 0
        assert off % 8 == 0
        off = (off + 9 * co * (c0 + c1) + 7) // 8 * 8
        assert off % 8 == 0
        off = (off + co + 7) // 8 * 8
        seen.append(name)
    assert len(seen) == 14 and len(set(seen)) == 14
    n_params = sum(9 * co * (c0 + c1) + co for _, c0, c1, co in LAYERS) + 17
    assert 480_000 < n_params < 500_000
