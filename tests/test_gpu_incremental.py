"""Incremental broadphase (cc_set_incremental): a moving scene stepped with a
kept candidate list gives, every step, exactly the outputs of full rebuilds —
through small moves (list kept), a large jump (rebuilt: the step that moved
too far is redone) and a scene that outgrows its grid."""
import numpy as np
import pytest
import torch

from collide_b200 import scenes as S
from collide_b200 import serving as SV

pytestmark = pytest.mark.gpu


def snap(p):
    P, C = p.n_pairs, p.n_contacts
    return (P, C, p.pairs[:P].cpu().numpy(), p.norm[:C].cpu().numpy().view(np.uint32),
            p.depth[:C].cpu().numpy().view(np.uint32), p.aabb.cpu().numpy().view(np.uint32))


def test_incremental_steps_equal_full_rebuilds(cb):
    m = S.mixed_slab(200_000, seed=8, extent=(3.0, 3.0, 0.3))
    dsa, dsb = cb.DeviceScene(m), cb.DeviceScene(m)
    ca, cb_ = cb.Context(), cb.Context()
    ca.set_incremental(True, 0.5)
    pa, pb = cb.DevicePipeline(dsa, ctx=ca), cb.DevicePipeline(dsb, ctx=cb_)
    plan = [1e-6] * 6 + [3e-2] + [1e-6] * 3 + ["grow"] + [1e-6] * 3
    kept = 0
    for step, move in enumerate(plan):
        for ds in (dsa, dsb):
            if move == "grow":  # the scene spreads beyond the kept grid
                ds.pos.mul_(1.25)
            else:
                SV.perturb_(ca, ds, 1000 + step, sigma=move, max_angle=1e-3)
        pa.run()
        pb.run()
        a, b = snap(pa), snap(pb)
        assert a[0] == b[0] and a[1] == b[1], (step, a[:2], b[:2])
        for x, y in zip(a[2:], b[2:]):
            assert np.array_equal(x, y), step
        kept += ca.last_step_rebuilt() == 0
    assert kept >= 5  # most small steps kept their lists


def test_incremental_redo_keeps_caller_boxes(cb):
    """A step that moved too far is redone from the caller's RECT and
    TRIANGLEMESH boxes (GenerateAABB leaves those to the caller): every shape
    type, boxes supplied before each step, equal to full rebuilds."""
    from test_gpu_shape_types import all_types_scene
    sc = all_types_scene(n=3000, seed=5)
    left = np.isin(sc.T, (S.RECT, S.TRIANGLEMESH))
    dsa, dsb = cb.DeviceScene(sc), cb.DeviceScene(sc)
    ca, cb_ = cb.Context(), cb.Context()
    ca.set_incremental(True, 1.0)
    # outputs large enough that no step is retried (a retry would see its RECT / TRIANGLEMESH boxes shifted)
    pa, pb = cb.DevicePipeline(dsa, ctx=ca, pairs_cap=400_000), cb.DevicePipeline(dsb, ctx=cb_, pairs_cap=400_000)
    rebuilt = []
    for step, move in enumerate([1e-6, 1e-6, 1e-6, 5e-2, 1e-6, 1e-6]):
        for ds, p in ((dsa, pa), (dsb, pb)):
            SV.perturb_(ca, ds, 500 + step, sigma=move, max_angle=1e-3)
            c = ds.pos.cpu().numpy()[sc.ID[left]]
            box = torch.zeros_like(p.aabb)
            box[:sc.n][torch.from_numpy(left)] = torch.from_numpy(c - 0.05).cuda()
            box[sc.n:][torch.from_numpy(left)] = torch.from_numpy(c + 0.05).cuda()
            p.aabb.copy_(box)
            p.run()
        a, b = snap(pa), snap(pb)
        assert a[0] == b[0] and a[1] == b[1], (step, a[:2], b[:2])
        for x, y in zip(a[2:], b[2:]):
            assert np.array_equal(x, y), step
        rebuilt.append(ca.last_step_rebuilt())
    assert rebuilt[0] == 1 and rebuilt[1] == 0 and rebuilt[3] == 1  # kept, then the jump was redone
