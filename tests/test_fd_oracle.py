"""CPU: the FP64 oracle's adjoint against FP64 central finite differences
(the differentiation-check workload: 2k Gaussians, 128x128, 200 random raw
parameters drawn with the FD seed).  At h=1e-6 the difference quotient is
local enough that the comparison is exact to ~1e-9; at the configured
h=1e-4 some quotients straddle an L1 kink or an alpha / transmittance
threshold, so the reference's own FD tolerance is applied
(tools/verify_gradients_extended.py:455-490)."""
import numpy as np

import gsutil as U
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O


def test_fp64_adjoint_matches_central_differences():
    w = S.config_fd_2k()
    sc, cam = w.scene, w.cameras[0]
    cfg = S.render_config(True)
    gt = O.forward(w.target_scene, cam, S.render_config(False), "c").image
    _, _, g64 = O.step_f64(sc, cam, cfg, gt)
    keys = ("pos", "sc", "rot", "sh", "op")
    p64 = [np.ascontiguousarray(x, np.float64).reshape(-1).copy() for x in
           (sc.positions, sc.scales, sc.rotations, sc.sh, sc.opacities)]
    rng = np.random.default_rng(S.SEED_FD)
    picks = []
    for _ in range(200):
        grp = int(rng.integers(5))
        picks.append((grp, int(rng.integers(len(p64[grp])))))
    ana = np.array([g64[keys[grp]][i] for grp, i in picks])
    for h, min_cos, min_within in ((1e-6, 1 - 1e-9, 1.0), (1e-4, 0.99, 0.95)):
        fd = []
        for grp, i in picks:
            o = p64[grp][i]
            p64[grp][i] = o + h
            lp, _, _ = O.step_f64(sc, cam, cfg, gt, want_grads=False, params64=p64)
            p64[grp][i] = o - h
            lm, _, _ = O.step_f64(sc, cam, cfg, gt, want_grads=False, params64=p64)
            p64[grp][i] = o
            fd.append((lp - lm) / (2 * h))
        fd = np.array(fd)
        assert U.cosine(fd, ana) >= min_cos, h
        within = np.abs(fd - ana) <= 5e-5 * np.abs(fd).max() + 0.10 * np.maximum(np.abs(fd), np.abs(ana))
        assert within.mean() >= min_within, h
