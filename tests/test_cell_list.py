"""The cell-list neighbour search's geometry (k_pair.cu: cell_axis, the 5 x 5 x 5 stencil),
restated in numpy: for random boxes, wrapped and unwrapped centres, every pair within the
list radius under the minimum image lies in the stencil of the first molecule's cell, and
the stencil's cells are distinct, so no candidate is visited twice."""
import numpy as np


def cell_axis(x, box, side, nc):
    p = x - box * np.floor(x / box)
    c = (p / side).astype(int)
    return np.clip(c, 0, nc - 1)


def test_stencil_covers_the_list_radius():
    rng = np.random.default_rng(3)
    for trial in range(40):
        rl = rng.uniform(6.0, 10.0)
        box = rl * rng.uniform(3.0, 6.0)
        nc = int(np.floor(2.0 * box / rl))
        assert nc >= 6
        side = box / nc
        n = 400
        x = rng.uniform(-box, 2 * box, (n, 3))  # centres need not be wrapped
        cell = np.stack([cell_axis(x[:, a], box, side, nc) for a in range(3)], axis=1)
        d = x[:, None, :] - x[None, :, :]
        d -= box * np.round(d / box)
        close = (d ** 2).sum(-1) < rl * rl
        dc = (cell[None, :, :] - cell[:, None, :]) % nc
        dc = np.minimum(dc, nc - dc)  # cyclic cell distance per axis
        inside = (dc <= 2).all(-1)
        assert not (close & ~inside).any(), trial
        offs = np.array([(t % 5 - 2, (t // 5) % 5 - 2, t // 25 - 2) for t in range(125)])
        for c0 in cell[:5]:
            cells = {tuple((c0 + o) % nc) for o in offs}
            assert len(cells) == 125
