"""CUDA path against the FP64 oracle and the reference's own outputs.

Tolerances (relative L2 unless stated):
* forward projector vs oracle FP64 and vs reference: 1e-5;
* backprojector (reference semantics, exact weights) vs oracle FP64: 1e-5;
  vs the reference's texture-filtered backprojector: 5e-4;
* adjoint mode: |<Ax,y> - <x,A^T y>| / |<Ax,y>| < 1e-6;
* PFDR vs oracle and reference: 1e-5; FBP vs oracle: 1e-5, vs reference 1e-3;
* RD/TV vs oracle and reference: 1e-5; MLEM vs oracle FP64: 1e-5 per
  iteration checked, vs reference call sequence: 2e-3 (texture weights).
"""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden, rel_l2
from helpers import oracle_geoms, product_geoms

pytestmark = pytest.mark.gpu

PROJ_CASES = ["g0", "g90", "g30", "gpitch", "gpetx", "g0t1"]


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("name", PROJ_CASES)
def test_forward_projection(cuda, name):
    from petl_b200 import ops
    z = load_golden(f"proj_{name}.npz")
    geoms, ogeoms = product_geoms(z), oracle_geoms(z)
    for key in ("f", "f_noise"):
        g = ops.project(geoms, _t(z[key], cuda))
        want = O.project(ogeoms, z[key])
        for i in range(len(geoms)):
            assert rel_l2(_np(g[i]), want[i]) < 1e-5
            ref = z[f"g{i}"] if key == "f" else z[f"gnoise{i}"]
            assert rel_l2(_np(g[i]), ref) < 1e-5


@pytest.mark.parametrize("name", PROJ_CASES)
def test_backprojection_reference_semantics(cuda, name):
    from petl_b200 import ops
    z = load_golden(f"proj_{name}.npz")
    geoms, ogeoms = product_geoms(z), oracle_geoms(z)
    ys = [z[f"y{i}"] for i in range(len(geoms))]
    f = ops.backproject(geoms, [_t(y, cuda) for y in ys])
    assert rel_l2(_np(f), O.backproject(ogeoms, ys)) < 1e-5
    assert rel_l2(_np(f), z["b"]) < 5e-4
    s = ops.backproject(geoms, [_t(np.ones(G.shape), cuda) for G in geoms])
    assert rel_l2(_np(s), z["sens"]) < 2e-4


@pytest.mark.parametrize("name", PROJ_CASES)
def test_adjoint_mode_is_exact_transpose(cuda, name):
    import torch
    from petl_b200 import ops
    z = load_golden(f"proj_{name}.npz")
    geoms = product_geoms(z)
    rng = np.random.default_rng(7)
    x = _t(rng.random(geoms[0].vol_shape), cuda)
    ys = [_t(rng.random(G.shape), cuda) for G in geoms]
    Ax = ops.project(geoms, x)
    Aty = ops.backproject(geoms, ys, mode="adjoint")
    lhs = sum(float(torch.sum(a.double() * y.double())) for a, y in zip(Ax, ys))
    rhs = float(torch.sum(x.double() * Aty.double()))
    assert abs(lhs - rhs) / abs(lhs) < 1e-6


def test_subsets_and_slabs_compose(cuda):
    import torch
    from petl_b200 import ops
    z = load_golden("proj_g0.npz")
    G = product_geoms(z)[0]
    f = _t(z["f"], cuda)
    full = ops.project(G, f)
    parts = torch.zeros_like(full)
    for s in range(3):
        ops.project(G, f, parts, subset=(s, 3))
    assert torch.equal(full, parts)
    slabs = torch.zeros_like(full)
    ops.project(G, f, slabs, v1_range=(0, 4))
    ops.project(G, f, slabs, v1_range=(4, G.shape[0]))
    assert torch.equal(full, slabs)
    y = _t(z["y0"], cuda)
    b = ops.backproject(G, y)
    b2 = ops.backproject(G, y, subset=(0, 2))
    ops.backproject(G, y, f=b2, subset=(1, 2), accumulate=True)
    assert rel_l2(_np(b2), _np(b)) < 1e-6
    b3 = ops.backproject(G, y, v1_range=(0, 3))
    ops.backproject(G, y, f=b3, v1_range=(3, G.shape[0]), accumulate=True)
    assert rel_l2(_np(b3), _np(b)) < 1e-6


def test_nnz_matches_oracle(cuda):
    from petl_b200 import ops
    for name in ("g0", "g30", "gpitch"):
        z = load_golden(f"proj_{name}.npz")
        # taps whose weight is exactly zero in one rounding and a few ulp in
        # another flip the count; float vs float agrees to a small fraction
        n_gpu = ops.nnz(product_geoms(z)[0])
        n_f32 = O.project_nnz(oracle_geoms(z)[0], single=True)
        assert abs(n_gpu - n_f32) / n_f32 < 2e-3, (n_gpu, n_f32)
        assert abs(n_gpu - O.project_nnz(oracle_geoms(z)[0])) / n_f32 < 3e-2


def test_cabi_host_path_matches_device_path(cuda):
    from petl_b200 import PETLserver, ops
    z = load_golden("proj_gpetx.npz")
    s = PETLserver()
    for p in z["planograms"]:
        psi, D, L, H, T, vm0, vm1 = p
        s.add_planogram(psi, D, L, H, T, vm0, vm1)
    s.set_volume(*[int(v) if i < 3 else float(v) for i, v in enumerate(z["volume"])])
    g = s.allocate_projections()
    s.project(g, z["f"].astype(np.float32))
    for i in range(2):
        assert rel_l2(g[i], z[f"g{i}"]) < 1e-5
    f = s.backproject([z["y0"].copy(), z["y1"].copy()])
    dev = ops.backproject(s.geometries_from_model(), [_t(z["y0"], cuda), _t(z["y1"], cuda)])
    assert rel_l2(f, _np(dev)) < 1e-6
    assert rel_l2(f, z["b"]) < 5e-4


@pytest.mark.parametrize("name", ["g0", "g0t1"])
def test_pfdr_ramp_fbp(cuda, name):
    from petl_b200 import PETLserver, ops
    z = load_golden(f"pfdr_{name}.npz")
    G, Go = product_geoms(z)[0], oracle_geoms(z)[0]
    g = _t(z["g"], cuda)
    reb = ops.pfdr(G, g)
    want = O.pfdr(Go, z["g"])
    assert rel_l2(_np(reb), want) < 1e-5
    assert rel_l2(_np(reb), z["g_reb"]) < 1e-5
    f = ops.fbp(G, g)
    assert rel_l2(_np(f), O.fbp(Go, z["g"])) < 1e-5
    assert rel_l2(_np(f), z["fbp"]) < 1e-3
    # through the reference C ABI: PFDR rewrites the model to N_v1 = 1
    s = PETLserver()
    psi, D, L, H, T, vm0, vm1 = z["planograms"][0]
    s.add_planogram(psi, D, L, H, T, vm0, vm1)
    s.set_volume(*[int(v) if i < 3 else float(v) for i, v in enumerate(z["volume"])])
    fb = s.FBP([z["g"].astype(np.float32).copy()])
    assert rel_l2(fb, z["fbp"]) < 1e-3
    gr = s.PFDR([z["g"].astype(np.float32).copy()])
    assert rel_l2(gr[0], z["g_reb"]) < 1e-5
    assert tuple(s.get_planogramSize(0)) == tuple(z["shape_after"])


def test_regularizers(cuda):
    from petl_b200 import PETLserver, ops
    r = load_golden("regularizers.npz")
    s = PETLserver()
    for tag in ("3d", "2d"):
        f, d = r[f"f_{tag}"], r[f"d_{tag}"]
        ft, dt = _t(f, cuda), _t(d, cuda)
        g = ops.rd_gradient(ft, 2.0, 0.01)
        assert rel_l2(_np(g), O.rd_gradient(f, 2.0, 0.01)) < 1e-5
        assert rel_l2(_np(g), r[f"rd_grad_{tag}"]) < 1e-5
        assert rel_l2(s.relative_differences_grad(f.copy(), 2.0, 0.01), r[f"rd_grad_{tag}"]) < 1e-5
        for delta, p in ((0.05, 1.0), (0.3, 1.2)):
            key = f"{tag}_d{delta}_p{p}"
            tg = ops.tv_gradient(ft, delta, 0.7, p)
            assert rel_l2(_np(tg), r[f"tv_grad_{key}"]) < 1e-5
            assert abs(float(ops.tv_cost(ft, delta, 0.7, p)) / r[f"tv_cost_{key}"] - 1) < 1e-5
            assert abs(float(ops.tv_quadform(ft, dt, delta, 0.7, p)) / r[f"tv_quad_{key}"] - 1) < 1e-5
            assert abs(s.TVcost(f.copy(), delta, 0.7, p) / r[f"tv_cost_{key}"] - 1) < 1e-5
        fd = f.copy()
        s.diffuse(fd, 0.05, 3, 1.0)
        assert rel_l2(fd, r[f"diffuse_{tag}"]) < 1e-5
        fn = f.copy()
        s.TV_denoise(fn, 0.05, 0.5, 3, 1.0)
        assert rel_l2(fn, r[f"tvdenoise_{tag}"]) < 1e-5


def test_mlem_matches_oracle_and_reference(cuda):
    from petl_b200 import recon
    z = load_golden("mlem_g0.npz")
    G, Go = product_geoms(z)[0], oracle_geoms(z)[0]
    g = _t(z["g"], cuda)
    for tag, beta in (("plain", 0.0), ("rd", 0.05)):
        f, _ = recon.mlem(G, g, 4, beta=beta, delta=2.0)
        assert rel_l2(_np(f), O.mlem(Go, z["g"], 4, beta=beta, delta=2.0)) < 1e-5
        assert rel_l2(_np(f), z[f"f_{tag}"][3]) < 2e-3


def test_mlem_with_response_matches_oracle(cuda):
    """A set response R makes MLEM's model R P (the reference's MLEM turns
    include_response_with_projectors on): device MLEM and OSEM against the
    oracle's literal restatement of the reference sequence, through
    recon.mlem and through PETLserver.MLEM after set_response."""
    from petl_b200 import PETLserver, recon
    z = load_golden("mlem_g0.npz")
    G, Go = product_geoms(z)[0], oracle_geoms(z)[0]
    rng = np.random.default_rng(21)
    R = O.solid_angle([Go], [rng.uniform(0.5, 1.0, size=Go.shape).astype(np.float32)], inverse=True)[0]
    R[rng.random(Go.shape) < 0.02] = 0.0
    want = O.mlem(Go, z["g"], 4, response=R)
    f, _ = recon.mlem(G, _t(z["g"], cuda), 4, response=[_t(R, cuda)])
    assert rel_l2(_np(f), want) < 1e-5
    # the response changes the result
    assert rel_l2(want, O.mlem(Go, z["g"], 4)) > 1e-3
    s = PETLserver()
    s.add_planogram(*z["planograms"][0])
    s.set_volume(*[int(v) if i < 3 else float(v) for i, v in enumerate(z["volume"][:5])])
    s.set_response([R])
    fs = s.MLEM([z["g"].astype(np.float32)], None, 4)
    assert rel_l2(fs, want) < 1e-5


def test_osem_one_subset_equals_mlem_and_matches_oracle(cuda):
    import torch
    from petl_b200 import recon
    z = load_golden("mlem_g0.npz")
    G, Go = product_geoms(z)[0], oracle_geoms(z)[0]
    g = _t(z["g"], cuda)
    a, _ = recon.mlem(G, g, 3)
    b, _ = recon.osem(G, g, 3, 1)
    assert torch.equal(a, b)
    c, hist = recon.osem(G, g, 2, 4, loglik_every=1)
    assert rel_l2(_np(c), O.osem(Go, z["g"], 2, 4)) < 1e-5
    assert float(hist[1]) > float(hist[0])


def test_gaussian_filter_matches_direct_formula(cuda):
    import torch
    from petl_b200 import ops
    rng = np.random.default_rng(3)
    f = rng.random((6, 9, 11)).astype(np.float32)
    out = _np(ops.gaussian_filter_(_t(f, cuda), 2.5, 3))
    # direct 3-D evaluation of the reference kernel (clamped-distance weights)
    sigma = 2.5 / (2 * np.sqrt(2 * np.log(2)))
    R = int(np.ceil(np.sqrt(2 * np.log(10)) * sigma))
    den = 1.0 / (2 * sigma)
    want = np.zeros_like(f, dtype=np.float64)
    N = f.shape
    for i in range(N[0]):
        for j in range(N[1]):
            for k in range(N[2]):
                val = s = 0.0
                for di in range(-R, R + 1):
                    ii = min(max(i + di, 0), N[0] - 1)
                    for dj in range(-R, R + 1):
                        jj = min(max(j + dj, 0), N[1] - 1)
                        for dk in range(-R, R + 1):
                            kk = min(max(k + dk, 0), N[2] - 1)
                            w = np.exp(-den * ((i - ii) ** 2 + (j - jj) ** 2 + (k - kk) ** 2))
                            val += w * f[ii, jj, kk]
                            s += w
                want[i, j, k] = val / s
    assert rel_l2(out, want) < 1e-5
    del torch


def test_rwls_matches_oracle(cuda):
    """PCG least squares (PETLserver.RWLS) on the device against the FP64
    oracle's restatement of the reference loop: plain, weighted with the SQS
    preconditioner, Huber-TV regularized, without the non-negativity
    constraint, and with a response in the projectors.  FP32 projections
    and FP64 reductions against FP64 throughout: 1e-4 relative L2 after 4
    iterations."""
    from petl_b200 import recon
    z = load_golden("mlem_g0.npz")
    G, Go = product_geoms(z)[0], oracle_geoms(z)[0]
    g = z["g"].astype(np.float32)
    W = (1.0 / np.maximum(g, 7.0)).astype(np.float32)
    rng = np.random.default_rng(9)
    R = rng.uniform(0.5, 1.0, size=g.shape).astype(np.float32)
    f0 = np.zeros(Go.vol_shape, np.float32)
    cases = [
        (dict(), dict()),
        (dict(W=[_t(W, cuda)], preconditioner="SQS"), dict(W=W, sqs=True)),
        (dict(delta=0.5, beta=0.02, preconditioner="SQS"), dict(delta=0.5, beta=0.02, sqs=True)),
        (dict(nonnegativity=False), dict(nonnegativity=False)),
        (dict(response=[_t(R, cuda)], W=[_t(W, cuda)]), dict(response=R, W=W)),
    ]
    for mine, theirs in cases:
        got = recon.rwls(G, _t(g, cuda), _t(f0, cuda), 4, **mine)
        want = O.rwls(Go, g, f0, 4, **theirs)
        assert rel_l2(_np(got), want) < 1e-4, (mine.keys(), rel_l2(_np(got), want))


def test_server_least_squares_family(cuda):
    """PETLserver.LS / RLS / WLS / RWLS against the oracle; RWLS with a set
    response not in the projectors corrects g in place, weights by the
    response squared and multiplies g back at the end, as the reference."""
    from petl_b200 import PETLserver, recon, ops
    z = load_golden("mlem_g0.npz")
    Go = oracle_geoms(z)[0]
    g = z["g"].astype(np.float32)
    s = PETLserver()
    s.add_planogram(*z["planograms"][0])
    s.set_volume(*[int(v) if i < 3 else float(v) for i, v in enumerate(z["volume"][:5])])
    f0 = np.zeros(Go.vol_shape, np.float32)
    assert rel_l2(s.LS([g.copy()], f0.copy(), 3), O.rwls(Go, g, f0, 3)) < 1e-4
    assert rel_l2(s.RLS([g.copy()], f0.copy(), 3, 0.5, 0.02, True),
                  O.rwls(Go, g, f0, 3, delta=0.5, beta=0.02, sqs=True)) < 1e-4
    # WLS with the default weights: 1 / max(gaussian(g), 7) from the device
    Wd = recon.auto_weights([_t(g, cuda)])[0]
    assert rel_l2(s.WLS([g.copy()], f0.copy(), 3), O.rwls(Go, g, f0, 3, W=_np(Wd))) < 1e-4
    # a response in the projectors
    rng = np.random.default_rng(4)
    R = rng.uniform(0.5, 1.0, size=g.shape).astype(np.float32)
    s.set_response([R])
    got = s.RWLS([g.copy()], f0.copy(), 3, W=[np.ones_like(g)], include_response_with_projectors=True)
    assert rel_l2(got, O.rwls(Go, g, f0, 3, W=np.ones_like(g), response=R)) < 1e-4
    # a response applied to the data
    gg = [g.copy()]
    got = s.RWLS(gg, f0.copy(), 3)
    gc = ops.apply_corrections_(s.geometries_from_model()[0], _t(g, cuda), _t(R, cuda), 0.75)
    assert np.array_equal(gg[0], _np(gc) * R)
    want = O.rwls(Go, _np(gc), f0, 3, W=_np(Wd) * R * R)
    assert rel_l2(got, want) < 1e-4


@pytest.mark.parametrize("num_dims", [1, 2, 3])
def test_gaussian_filter_against_reference(cuda, num_dims):
    """gaussian_filter (src/relative_differences.cu:314-411,753-800) along 1, 2
    and 3 dimensions at the widths the reference's Python layer uses, on the
    device path and through the C ABI."""
    from petl_b200 import PETLserver, ops
    z = load_golden("gaussian.npz")
    s = PETLserver()
    s.add_planogram(0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25)
    for fwhm in (0.6571, 2.0, 3.0):
        f = z[f"in_{num_dims}_{fwhm}"]
        want = z[f"out_{num_dims}_{fwhm}"]
        got = _np(ops.gaussian_filter_(_t(f, cuda), fwhm, num_dims))
        assert rel_l2(got, want) < 1e-5, fwhm
        h = f.copy()
        s.gaussian_filter(h, fwhm, num_dims)
        assert rel_l2(h, want) < 1e-5, fwhm
