"""The scan formulation of inpainting (tests/inpaint_model.py, which the CUDA
inpainting kernels implement) against the oracle's literal Gauss-Seidel
sweeps (inpainting.cpp:104-136) on random hole masks, including the edge
cases the sweeps have: no hole, all holes but one pixel, holes on every
border, single-row and single-column images."""
import numpy as np
import pytest

import oracle as O
from inpaint_model import inpaint_sources


def _oracle_sources(hole):
    h, w = hole.shape
    q = np.where(hole, 0.0, 1.0).astype(np.float32)
    color = np.zeros((h, w, 3), np.float32)
    out, src, sweeps = O.inpaint(color, q)
    return src, sweeps


def _masks():
    rng = np.random.default_rng(1234)
    yield "none", np.zeros((9, 13), bool)
    m = np.ones((11, 7), bool)
    m[5, 3] = False
    yield "single_source", m
    m = np.zeros((16, 20), bool)
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = True
    yield "border", m
    yield "row", rng.random((1, 40)) < 0.5
    yield "column", rng.random((40, 1)) < 0.5
    for k, (h, w, p) in enumerate([(24, 32, 0.3), (37, 53, 0.6), (64, 48, 0.85), (30, 90, 0.95)]):
        m = rng.random((h, w)) < p
        if m.all():
            m[h // 2, w // 2] = False
        yield f"random{k}", m
    # blobs: rectangles of holes (disocclusions)
    m = np.zeros((60, 80), bool)
    for _ in range(12):
        y, x = rng.integers(0, 60), rng.integers(0, 80)
        m[y:y + rng.integers(2, 20), x:x + rng.integers(2, 30)] = True
    yield "blobs", m


@pytest.mark.parametrize("name,hole", list(_masks()), ids=[n for n, _ in _masks()])
def test_scan_model_matches_sweeps(name, hole):
    src, sweeps = _oracle_sources(hole)
    model = inpaint_sources(hole)
    np.testing.assert_array_equal(model[hole], src[hole])
    assert sweeps <= 3


def test_inpaint_copies_colour_of_source():
    rng = np.random.default_rng(5)
    h, w = 20, 30
    hole = rng.random((h, w)) < 0.4
    q = np.where(hole, 0.0, 1.0).astype(np.float32)
    color = rng.random((h, w, 3)).astype(np.float32)
    out, src, _ = O.inpaint(color, q)
    np.testing.assert_array_equal(out[~hole], color[~hole])
    ys, xs = np.nonzero(hole)
    np.testing.assert_array_equal(out[ys, xs], color[src[ys, xs, 1], src[ys, xs, 0]])
