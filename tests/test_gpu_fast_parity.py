"""Parity of the benched (fast-rounding) build with the CPU oracle, on a B200.

The fast build contracts multiply-adds, divides and takes square roots approximately
(IEEE kept where a decision or a compared direction depends on it), and replaces the
Stokes rotation's and the TIR retarder's atan2 / sincos by double-angle identities.  The
reference's GPU equivalence harness holds its GPU port to per-function ULP budgets
(crates/indicatrix/docs/gpu_harness_last_run.json:29-72, the hybrid ULP-or-absolute-floor
rule of renderer/gpu/ulp.rs:33-42) and to per-pixel z statistics over disjoint sample
ranges (renderer/gpu/z_stats.rs:95-110).  The same bars are applied here to both builds,
on the benchmark's own inputs: the seeded random stones (Cauchy and Sellmeier-1, n_D up
to 2.60, spline absorption, tilts 0-40 degrees), traced by the kernels the benchmark
times.
"""
import ctypes as C

import numpy as np
import pytest

from indicatrix_b200 import abi, materials, workloads
from indicatrix_b200.backend import BatchPlan

pytestmark = pytest.mark.gpu

CHECK_DISPERSION, CHECK_CMF, CHECK_EXP_LANE = 2, 3, 5
CHECK_TRACE, CHECK_ABSORPTION = 10, 12
CHECK_STOKES_ROTATE, CHECK_FRESNEL_CHANNEL, CHECK_CHANNEL_ALPHA = 14, 15, 16

# The reference's Tier-2 budgets (gpu_harness_last_run.json) and each check's absolute
# floor (renderer/gpu/environment_check/cmf.rs:34, transport_check/dispersion.rs:24,
# frame_and_tir.rs:45, :130, :192, fresnel.rs:28, :120, absorption_pleochroism.rs:60, :238).
BUDGET = {"dispersion": 24, "spectral_absorption": 24, "cmf": 32, "frame_rotation": 16,
          "signed_frame_rotation_psi": 32, "fresnel_reflection": 16, "fresnel_transmission": 16,
          "tir_retardation": 16, "pleochroic_channel_alpha": 48}
FLOOR = {"dispersion": 1e-6, "spectral_absorption": 1e-6, "cmf": 1e-6, "frame_rotation": 1e-6,
         "signed_frame_rotation_psi": 1e-5, "fresnel_reflection": 1e-6, "fresnel_transmission": 1e-6,
         "tir_retardation": 1e-6, "pleochroic_channel_alpha": 1e-5}


def ulp_diff(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, np.int64(-2**31) - a, a)
    b = np.where(b < 0, np.int64(-2**31) - b, b)
    return np.abs(a - b)


def within(got, want, budget, floor):
    """ulp.rs within_tolerance: ULP distance within the budget, or an absolute difference
    below the floor (values at or crossing zero)."""
    got = np.asarray(got, np.float32)
    want = np.asarray(want, np.float32)
    return (ulp_diff(got, want) <= budget) | (np.abs(got.astype(np.float64) - want.astype(np.float64)) < floor)


def bench_stones(n=8):
    return workloads.random_stones(64)[:n]


def scene_with(material, w=16, h=16):
    fs = workloads.round_brilliant_frame(w, h)
    fs.material = material
    return fs


@pytest.fixture(params=["exact", "fast"])
def build(request, backend, exact_backend):
    return request.param, (exact_backend if request.param == "exact" else backend)


def test_dispersion_and_cmf_budgets(build, oracle):
    """DispersionModel::evaluate (24 ULP) for the Diamond Sellmeier, and the bench stones'
    Cauchy and Sellmeier-1 fits; cie_1931_cmf (32 ULP).  Exact build: bit-exact."""
    name, b = build
    rng = np.random.default_rng(21)
    lam = np.concatenate([np.float32([380.0, 555.0, 779.9999, 486.1, 589.3, 656.3]),
                          rng.uniform(380.0, 780.0, 3000).astype(np.float32)])
    mats = [materials.diamond()] + [st.material for st in bench_stones(8)]
    kinds = set()
    for mat in mats:
        kinds.add(int(mat.dispersion.kind))
        out = b.debug_check(scene_with(mat), CHECK_DISPERSION, lam, 1).view(np.float32)[:, 0]
        want = np.array([oracle.lib().ixo_dispersion_eval(C.byref(mat.dispersion), float(x)) for x in lam],
                        np.float32)
        if name == "exact":
            assert np.array_equal(out.view(np.uint32), want.view(np.uint32))
        else:
            assert np.all(within(out, want, BUDGET["dispersion"], FLOOR["dispersion"])), ulp_diff(out, want).max()
    assert {abi.DISP_SELLMEIER1, abi.DISP_SELLMEIER3, abi.DISP_CAUCHY} <= kinds
    out = b.debug_check(scene_with(mats[0]), CHECK_CMF, lam, 3).view(np.float32)
    want = np.zeros((lam.size, 3), np.float32)
    for i, x in enumerate(lam):
        oracle.lib().ixo_cmf(float(x), oracle._f32p(want[i]))
    if name == "exact":
        assert np.array_equal(out.view(np.uint32), want.view(np.uint32))
    else:
        # absolute floor: the Gaussian tails (~1e-24), as the reference's cmf check uses
        assert np.all(within(out, want, BUDGET["cmf"], FLOOR["cmf"])), ulp_diff(out, want).max()


def test_exp_lane_bit_exact_in_both_builds(build, oracle):
    """exp_lane / exp_f32x8 (simd/exp_poly.rs:37): the Cephes polynomial with the
    reference's constants and clamp rule is bit-exact in both builds."""
    _, b = build
    rng = np.random.default_rng(5)
    xs = np.concatenate([rng.uniform(-90, 12, 4000), [0.0, -0.0, np.nan, np.inf, -np.inf, -87.5, 88.5]]
                        ).astype(np.float32)
    out = b.debug_check(scene_with(materials.diamond()), CHECK_EXP_LANE, xs, 1).view(np.float32)[:, 0]
    want = np.array([oracle.lib().ixo_exp_lane(float(x)) for x in xs], np.float32)
    assert np.array_equal(out.view(np.uint32), want.view(np.uint32))


def test_spline_absorption_matches_oracle(build, oracle):
    """spectral_absorption of the bench stones' 16-knot splines (0-5 /cm) and a stress
    spline (0-8 /cm): bit-exact in the exact build, within 24 ULP in the fast build."""
    name, b = build
    rng = np.random.default_rng(33)
    lam = np.concatenate([np.float32([380.0, 380.0001, 406.6667, 500.0, 779.99, 780.0]),
                          rng.uniform(380.0, 780.0, 2000).astype(np.float32)])
    mats = [st.material for st in bench_stones(8) if st.material.abs_o.has_spline]
    mats.append(workloads.stress_material())
    assert len(mats) >= 4
    for mat in mats:
        out = b.debug_check(scene_with(mat), CHECK_ABSORPTION, lam, 1).view(np.float32)[:, 0]
        want = np.array([oracle.lib().ixo_spectral_absorption(C.byref(mat.abs_o), float(x)) for x in lam],
                        np.float32)
        assert np.all(want >= 0.0) and want.max() > 0.0
        if name == "exact":
            assert np.array_equal(out.view(np.uint32), want.view(np.uint32))
        else:
            assert np.all(within(out, want, BUDGET["spectral_absorption"], FLOOR["spectral_absorption"])), \
                ulp_diff(out, want).max()


def unit(v):
    return (v / np.linalg.norm(v, axis=-1, keepdims=True)).astype(np.float32)


def test_stokes_rotation_to_plane_of_incidence(build, oracle):
    """rotate_stokes_to_plane_of_incidence (raytracer/absorption.rs:69): the rotated
    Stokes vector within frame_rotation + apply_matrix's 16 ULP (floor 1e-6), the new plane
    normal within the signed-psi check's 32 ULP (floor 1e-5).  The fast build forms cos 2psi / sin 2psi
    by double-angle identities instead of atan2 + sincos."""
    name, b = build
    rng = np.random.default_rng(44)
    n = 4000
    k = unit(rng.normal(size=(n, 3)))
    nrm = unit(rng.normal(size=(n, 3)))
    # The previous plane normal is perpendicular to the ray, as in transport: it is
    # normalize(k_prev x n_prev), and the new k lies in the plane of k_prev and n_prev.
    prev = unit(np.cross(k, rng.normal(size=(n, 3))))
    has_prev = (rng.uniform(size=n) < 0.9).astype(np.uint32)
    st = rng.uniform(-1, 1, (n, 4)).astype(np.float32)
    st[:, 0] = np.abs(st[:, 0]) + 0.5
    # edge rows: k along the normal (no plane), a degenerate previous plane
    nrm[:8] = k[:8]
    prev[8:16] = 0.0
    inp = np.concatenate([k, nrm, prev, has_prev.view(np.float32)[:, None], st], axis=1).astype(np.float32)
    out = b.debug_check(scene_with(materials.diamond()), CHECK_STOKES_ROTATE, inp, 7).view(np.float32)
    want_s = np.zeros((n, 4), np.float32)
    want_c = np.zeros((n, 3), np.float32)
    for i in range(n):
        oracle.lib().ixo_rotate_stokes(oracle._f32p(k[i].copy()), oracle._f32p(nrm[i].copy()),
                                       oracle._f32p(prev[i].copy()), int(has_prev[i]), oracle._f32p(st[i].copy()),
                                       oracle._f32p(want_s[i]), oracle._f32p(want_c[i]))
    ok_s = within(out[:, :4], want_s, BUDGET["frame_rotation"], FLOOR["frame_rotation"])
    ok_c = within(out[:, 4:], want_c, BUDGET["signed_frame_rotation_psi"], FLOOR["signed_frame_rotation_psi"])
    assert np.all(ok_s), ulp_diff(out[:, :4], want_s)[~ok_s].max()
    assert np.all(ok_c), ulp_diff(out[:, 4:], want_c)[~ok_c].max()
    if name == "exact":
        # no transcendental in the plane normal: the oracle's bits
        assert np.array_equal(out[:, 4:].view(np.uint32), want_c.view(np.uint32))


def test_fresnel_reflection_transmission_and_tir(build, oracle):
    """One channel's Fresnel step, inside and outside, across the bench's index range:
    reflected Stokes (fresnel_reflection + apply_matrix, 16 ULP; the TIR retarder,
    tir_retardation + apply_matrix, 16 ULP), transmitted Stokes (fresnel_transmission +
    apply_matrix, 16 ULP) and r_s, r_p, t_s, t_p (16 ULP), each with the reference's
    absolute floor of 1e-6 for values at a zero crossing (Brewster's angle); TIR decided
    identically."""
    name, b = build
    rng = np.random.default_rng(55)
    n = 6000
    n_idx = rng.uniform(1.45, 2.7, n).astype(np.float32)
    inside = rng.uniform(size=n) < 0.5
    n1 = np.where(inside, n_idx, np.float32(1.0)).astype(np.float32)
    n2 = np.where(inside, np.float32(1.0), n_idx).astype(np.float32)
    cos_i = rng.uniform(0.0, 1.0, n).astype(np.float32)
    cos_i[:6] = [0.0, 1.0, 1e-7, 0.999999, 0.5, 0.25]
    st = rng.uniform(-1, 1, (n, 4)).astype(np.float32)
    st[:, 0] = np.abs(st[:, 0]) + 1.0
    inp = np.concatenate([np.stack([n1, n2, cos_i], axis=1), st], axis=1).astype(np.float32)
    out = b.debug_check(scene_with(materials.diamond()), CHECK_FRESNEL_CHANNEL, inp, 13).view(np.float32)
    want = np.zeros((n, 13), np.float32)
    for i in range(n):
        oracle.lib().ixo_fresnel_channel(float(n1[i]), float(n2[i]), float(cos_i[i]), oracle._f32p(st[i].copy()),
                                         oracle._f32p(want[i]))
    assert np.array_equal(out[:, 12], want[:, 12])
    tir = want[:, 12] > 0
    assert 0.05 < tir.mean() < 0.5
    ok_tir = within(out[:, :4], want[:, :4], BUDGET["tir_retardation"], FLOOR["tir_retardation"])
    ok_r = within(out[:, :4], want[:, :4], BUDGET["fresnel_reflection"], FLOOR["fresnel_reflection"])
    assert np.all(ok_tir[tir]), ulp_diff(out[tir, :4], want[tir, :4]).max()
    assert np.all(ok_r[~tir]), ulp_diff(out[~tir, :4], want[~tir, :4]).max()
    ok_t = within(out[~tir, 4:8], want[~tir, 4:8], BUDGET["fresnel_transmission"], FLOOR["fresnel_transmission"])
    assert np.all(ok_t), ulp_diff(out[~tir, 4:8], want[~tir, 4:8]).max()
    ok_c = within(out[~tir, 8:12], want[~tir, 8:12], BUDGET["fresnel_transmission"], FLOOR["fresnel_transmission"])
    assert np.all(ok_c), ulp_diff(out[~tir, 8:12], want[~tir, 8:12]).max()
    if name == "exact":
        # no transcendental outside TIR: the reflection and transmission round as the
        # oracle (0 ULP; +0 and -0 are one value, as ulp.rs counts them)
        assert ulp_diff(out[~tir, :12], want[~tir, :12]).max() == 0


def test_isotropic_channel_alpha(build, oracle):
    """channel_absorption_alphas_assigned's non-birefringent branch
    (raytracer/absorption.rs:197): the midpoint of the tensor's quadratic form over the two
    eigen-polarisations, on the bench stones' splines, within the pleochroic alpha budget
    (48 ULP); bit-exact in the exact build."""
    name, b = build
    rng = np.random.default_rng(66)
    n = 3000
    k = unit(rng.normal(size=(n, 3)))
    k[0] = [0.0, 1.0, 0.0]  # along the default optic axis: the degenerate basis
    lam = rng.uniform(380, 780, n).astype(np.float32)
    inp = np.concatenate([k, lam[:, None]], axis=1).astype(np.float32)
    for st in [s for s in bench_stones(8) if s.material.abs_o.has_spline][:3]:
        mat = st.material
        out = b.debug_check(scene_with(mat), CHECK_CHANNEL_ALPHA, inp, 1).view(np.float32)[:, 0]
        want = np.array([oracle.lib().ixo_channel_alpha(C.byref(mat), oracle._f32p(k[i].copy()), float(lam[i]))
                         for i in range(n)], np.float32)
        if name == "exact":
            assert np.array_equal(out.view(np.uint32), want.view(np.uint32))
        else:
            assert np.all(within(out, want, BUDGET["pleochroic_channel_alpha"], FLOOR["pleochroic_channel_alpha"])), \
                ulp_diff(out, want).max()


# ------------------------------------------------------------------------------------
# Per path and per pixel, on the benchmark's stones.
# ------------------------------------------------------------------------------------
def stone_scenes(w, h, picks=((0, 0.0), (1, 20.0), (2, 40.0), (3, 10.0), (5, 30.0))):
    stones = bench_stones(8)
    return [(i, t, workloads.tilted_scene(stones[i], t, w, h), stones[i]) for i, t in picks]


def trace_paths(b, fs, pixels, samples):
    inp = np.stack([pixels.astype(np.uint32), samples.astype(np.uint32)], axis=1)
    out = b.debug_check(fs, CHECK_TRACE, inp, 4)
    return out[:, :3].copy().view(np.float32), out[:, 3]


# Per-path agreement bars of the fast build on the bench stones (fractions of paths).
PATH_BARS = (0.85, 0.93, 0.93)


def test_fast_build_paths_on_bench_stones(backend, oracle):
    """Per-path XYZ of the fast build against the oracle on identical (pixel, sample)
    inputs, on bench stones of both dispersion forms, absorbing and clear, at several
    tilts.  A few-ULP difference can move a Fresnel / roulette draw across its threshold,
    after which a path legitimately differs, so the bars (PATH_BARS) are on fractions of
    paths: within 1e-4 relative, within 1e-2, and the same bounce count; the total within
    1 %."""
    W = H = 24
    spp = 16
    stats = []
    for idx, tilt, fs, st in stone_scenes(W, H):
        sc = fs.to_abi()
        xyz_o, bounces_o = oracle.trace_samples(sc, 0, W * H, 0, spp)
        px = np.repeat(np.arange(W * H), spp)
        sm = np.tile(np.arange(spp), W * H)
        xyz_g, bounces_g = trace_paths(backend, fs, px, sm)
        xo = xyz_o.reshape(-1, 3).astype(np.float64)
        xg = xyz_g.astype(np.float64)
        scale = np.maximum(np.abs(xo).max(axis=1), 1e-3)
        rel = np.abs(xg - xo).max(axis=1) / scale
        s = (np.mean(rel <= 1e-4), np.mean(rel <= 1e-2), np.mean(bounces_g == bounces_o.ravel()))
        stats.append(s)
        assert s[0] >= PATH_BARS[0] and s[1] >= PATH_BARS[1] and s[2] >= PATH_BARS[2], (idx, tilt, s)
        assert abs(xg.sum() - xo.sum()) <= 1e-2 * max(xo.sum(), 1e-6), (idx, tilt)
    print("per-path agreement (1e-4, 1e-2, bounces):", np.round(np.array(stats), 4).tolist())


def z_components(mean_a, se2_a, mean_b, se2_b):
    se2 = se2_a + se2_b
    z = np.zeros_like(mean_a)
    live = se2 > 0.0
    z[live] = (mean_b[live] - mean_a[live]) / np.sqrt(se2[live])
    return z


def largest_cluster(flags):
    """4-connected component sizes of flagged pixels (z_stats.rs connected_components)."""
    h, w = flags.shape
    seen = np.zeros_like(flags)
    best = 0
    for y in range(h):
        for x in range(w):
            if flags[y, x] and not seen[y, x]:
                stack, size = [(y, x)], 0
                seen[y, x] = True
                while stack:
                    cy, cx = stack.pop()
                    size += 1
                    for ny, nx in ((cy + 1, cx), (cy - 1, cx), (cy, cx + 1), (cy, cx - 1)):
                        if 0 <= ny < h and 0 <= nx < w and flags[ny, nx] and not seen[ny, nx]:
                            seen[ny, nx] = True
                            stack.append((ny, nx))
                best = max(best, size)
    return best


def passes_z_criteria(z, w, h):
    """z_stats.rs:95-110: |z| > 3 count <= max(5 * 0.0027 * N, 10) and no 4-connected
    cluster of such pixels larger than 6."""
    flags = (np.abs(z) > 3.0).reshape(h, w)
    count = int(flags.sum())
    cluster = largest_cluster(flags)
    return count <= max(5 * 0.0027 * w * h, 10) and cluster <= 6, count, cluster


def oracle_moments(oracle, sc, n_pix, first, spp):
    xyz, _ = oracle.trace_samples(sc, 0, n_pix, first, spp)
    x = xyz.astype(np.float64)
    return x.mean(axis=1), x.var(axis=1, ddof=1) / spp


TIER3_W = TIER3_H = 48
TIER3_SPP = 500


def test_tier3_fast_build_per_path_x_y_z(backend, oracle):
    """Tier 3 (z_stats.rs, estimator_check/image_comparison.rs): 48 x 48 px at 500 spp
    per side over disjoint absolute sample ranges -- the fast build's paths [0, 500) by
    the per-path check kernel, the oracle's [500, 1000) -- moments per pixel, z per pixel
    for each of X, Y and Z, and the reference's pass rule on each."""
    W, H, N = TIER3_W, TIER3_H, TIER3_SPP
    cases = [("diamond frame", workloads.round_brilliant_frame(W, H))]
    cases += [(f"stone {i} tilt {t}", fs) for i, t, fs, _ in stone_scenes(W, H, ((1, 20.0), (2, 40.0)))]
    for label, fs in cases:
        sc = fs.to_abi()
        mo, so = oracle_moments(oracle, sc, W * H, N, N)
        px = np.repeat(np.arange(W * H), N)
        sm = np.tile(np.arange(N), W * H)
        xyz_g, _ = trace_paths(backend, fs, px, sm)
        g = xyz_g.astype(np.float64).reshape(W * H, N, 3)
        mg, sg = g.mean(axis=1), g.var(axis=1, ddof=1) / N
        for c, name in enumerate("XYZ"):
            z = z_components(mo[:, c], so[:, c], mg[:, c], sg[:, c])
            ok, count, cluster = passes_z_criteria(z, W, H)
            assert ok, (label, name, count, cluster)


@pytest.mark.parametrize("variant", [2, 5, 8, 11])
def test_tier3_benched_batch_kernel(backend, oracle, variant):
    """Tier 3 on the kernel the benchmark times: a batch plan of bench stones (one
    persistent launch; the static task loop, or the path-pool loop at 128 / 64 / 256
    threads) traces samples [0, 500) of each 48 x 48 frame; the oracle traces [500, 1000).
    The plan returns sums, not samples, so each pixel's standard error uses the oracle's
    sample variance for both sides (the two estimators share one distribution under the
    null).  The reference's pass rule on X, Y and Z of every frame."""
    W, H, N = TIER3_W, TIER3_H, TIER3_SPP
    scenes = stone_scenes(W, H, ((1, 20.0), (4, 0.0), (6, 35.0)))
    plan = BatchPlan(backend, [(fs, 0, N) for _, _, fs, _ in scenes])
    if not plan.set_variant(variant):
        plan.close()
        pytest.skip(f"variant {variant} not in this build")
    plan.run()
    out = plan.download()
    for j, (idx, tilt, fs, _) in enumerate(scenes):
        mg = plan.sums(j).reshape(-1, 3) / N
        mo, so = oracle_moments(oracle, fs.to_abi(), W * H, N, N)
        for c, name in enumerate("XYZ"):
            z = z_components(mo[:, c], so[:, c], mg[:, c], so[:, c])
            ok, count, cluster = passes_z_criteria(z, W, H)
            assert ok, (variant, idx, tilt, name, count, cluster)
    assert np.all(np.isfinite(out))
    plan.close()
