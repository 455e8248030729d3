"""Gauss-point shape functions on the device (mel_mls_shapes) against the host restatement of the
pre-processor's MLS pass (generator.mls_shape: Preprocessor/MLS2DWithDerivatives.m:65-165,
WeightW1WithDerivatives.m:17-47, SupportDomain.m:16-18), and against the properties every linear
MLS basis has whatever the arithmetic: partition of unity and linear reproduction of N, and the
matching conditions on dN/dx, dN/dy."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the host solves the moment system in the pre-processor's global basis, whose conditioning
# (supports ~0.1 mm around points ~1 mm from the origin) leaves ~1e-10 relative error; the device
# solves a point-centred, scaled basis
TOL_HOST = 1e-8
TOL_REPRO = 1e-11


def _bodies(n=12, seed=4):
    from melody2d_b200 import generator as g
    sc = g.biaxial_scene(seed=seed, n_discs=n, workers=1)
    return [b for b in sc.bodies if b.kind == "deformable"]


def _check_reproduction(pts, nodes, csr, what):
    ptr, idx, N, Nx, Ny = csr
    P = len(ptr) - 1
    row = np.repeat(np.arange(P), np.diff(ptr))
    xs, ys = nodes[idx, 0] - pts[row, 0], nodes[idx, 1] - pts[row, 1]
    h = np.abs(xs).max()
    sums = lambda v: np.bincount(row, weights=v, minlength=P)
    # sum N = 1, sum N (x_i - x_p) = 0, sum dN/dx = 0, sum dN/dx (x_i - x_p) = 1, ...
    assert np.abs(sums(N) - 1).max() < TOL_REPRO, what
    assert np.abs(sums(N * xs)).max() < TOL_REPRO * h, what
    assert np.abs(sums(N * ys)).max() < TOL_REPRO * h, what
    scale = np.abs(Nx).max()
    assert np.abs(sums(Nx)).max() < TOL_REPRO * scale, what
    assert np.abs(sums(Ny)).max() < TOL_REPRO * scale, what
    assert np.abs(sums(Nx * xs) - 1).max() < TOL_REPRO * scale * h, what
    assert np.abs(sums(Ny * ys) - 1).max() < TOL_REPRO * scale * h, what
    assert np.abs(sums(Nx * ys)).max() < TOL_REPRO * scale * h, what


def test_mls_matches_host_and_reproduces_linear_fields(gpu_lib):
    from melody2d_b200.solver import mls_shapes
    bodies = _bodies()
    jobs = [(b.gp_xy, b.nodes, b.domain) for b in bodies] + [(b.nodes, b.nodes, b.domain) for b in bodies]
    host = [b.gp for b in bodies] + [b.sup for b in bodies]
    dev = mls_shapes(jobs)
    for k, ((pts, nodes, _), h, d) in enumerate(zip(jobs, host, dev)):
        np.testing.assert_array_equal(d[0], h[0])          # same support counts
        np.testing.assert_array_equal(d[1], h[1])          # same supports, ascending
        for a, b_, name in ((d[2], h[2], "N"), (d[3], h[3], "dNdx"), (d[4], h[4], "dNdy")):
            scale = np.abs(b_).max()
            assert np.abs(a - b_).max() <= TOL_HOST * scale, (k, name, np.abs(a - b_).max() / scale)
        _check_reproduction(pts, nodes, d, k)


def test_mls_singular_point_is_reported(gpu_lib):
    from melody2d_b200.solver import MelError, mls_shapes
    nodes = np.array([[0.0, 0.0], [1.0, 0.0], [2.0, 0.0], [3.0, 0.0]])   # collinear supports only
    radii = np.full(4, 1.5)
    pts = np.array([[1.5, 0.0]])
    with pytest.raises(MelError) as e:
        mls_shapes([(pts, nodes, radii)])
    assert "singular" in str(e.value)
