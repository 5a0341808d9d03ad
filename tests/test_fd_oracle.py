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
    picks = U.fd_picks([len(x) for x in p64], seed=S.SEED_FD)
    ana = np.array([g64[keys[grp]][i] for grp, i in picks])
    # h=1e-6: local quotients, exact agreement; h=1e-4 (the configured step):
    # quotients that straddle an L1 kink or a threshold are outliers, so the
    # reference tooling's per-element tolerance is the criterion there
    for h, min_cos, min_within in ((1e-6, 1 - 1e-9, 1.0), (1e-4, None, 0.95)):
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
        if min_cos is not None:
            assert U.cosine(fd, ana) >= min_cos, h
        assert U.fd_within(fd, ana).mean() >= min_within, h
