"""Host-side checks of the synthetic two-level box list
(camr_b200/problems.py `amr_box_list`) that the two-level workload and the
batched comparison run on: the boxes are disjoint, aligned, inside the fine
domain and coarse-aligned (even low corners, odd high corners, as
camr_amr_create requires), every drawn size comes from the stated set, and
the default configuration (350 boxes on the 512^3 fine index space of a
256^3 base) holds the 18,248,192 fine cells its measurements quote."""
import numpy as np

from camr_b200 import problems as P


def _check(boxes, fine_n, sizes, align):
    occ = np.zeros((fine_n,) * 3, dtype=np.int16)
    for lo, hi in boxes:
        lo, hi = np.array(lo), np.array(hi)
        ext = hi - lo + 1
        assert np.all(lo >= 0) and np.all(hi < fine_n)
        assert np.all(lo % align == 0)
        assert np.all(lo % 2 == 0) and np.all(hi % 2 == 1)
        assert all(int(e) in sizes for e in ext)
        occ[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] += 1
    assert occ.max() <= 1, "boxes overlap"
    return int(occ.sum())


def test_small_box_list_is_disjoint_aligned_and_drawn_from_sizes():
    sizes = (8, 16, 24)
    boxes = P.amr_box_list(nbox=24, fine_n=96, sizes=sizes, seed=3, align=8)
    assert len(boxes) == 24
    cells = _check(boxes, 96, sizes, 8)
    assert cells == sum(int(np.prod(np.array(h) - np.array(l) + 1)) for l, h in boxes)


def test_default_two_level_box_list():
    sizes = (16, 24, 32, 48, 64)
    boxes = P.amr_box_list(nbox=350, fine_n=512)
    assert len(boxes) == 350
    cells = _check(boxes, 512, sizes, 8)
    assert cells == 18_248_192
    # the drawn sizes keep the stated distribution: every size is used in
    # every direction, none dominates
    ext = np.array([np.array(h) - np.array(l) + 1 for l, h in boxes])
    for d in range(3):
        counts = [int((ext[:, d] == s).sum()) for s in sizes]
        assert min(counts) > 0.1 * 350 and max(counts) < 0.35 * 350


def test_box_list_is_reproducible():
    a = P.amr_box_list(nbox=40, fine_n=128, seed=7)
    b = P.amr_box_list(nbox=40, fine_n=128, seed=7)
    assert a == b
