"""Generate golden vectors by running the reference's own step math.

Run from the repository root, in a container that has the beamz source tree:

    python -m tests.golden.make_golden [--reference /path/to/beamz]

It loads beamz's source files by path under a numpy stand-in for ``jax``
(``_jaxshim.py``; JAX's x64-disabled dtype policy) and evaluates, on seeded
inputs, the reference functions that make up the leapfrog step:

* ``beamz/simulation/kernels.py``: ``cpml_coefficients`` (130), ``compile_cpml_term``
  (238), ``cpml_update_h_from_e_3d`` (458), ``cpml_update_e_from_h_3d`` (554),
  ``fused_update_h/e_lossy_3d_material`` (267/326), the 2D TM/TE curls (731-877)
  and ``precompute_h/e_update_coefficients`` (704-728);
* ``beamz/lattice.py``: ``sample_voxel_grid_at_e_component_3d_centered`` (732),
  ``_component_plane_plan_3d`` (274), ``sample_voxel_grid_at_component_2d`` (935);
* ``beamz/devices/_boundary_compile.py``: ``_compute_fdtdx_staggered_profile_1d``
  (479), ``compile_metallic_masks`` (118);
* ``beamz/devices/sources/time.py``: ``GaussianPulse.sample`` (459);
* ``beamz/simulation/observe.py``: ``_accumulate_dft`` (529) and its gate (327).

Multi-step fixtures compose those reference functions in the phase order of
``beamz/simulation/execute.py:467-541`` (pre-E sources, H, H sources, H PEC,
E, E sources, E PEC, DFT at t+dt, FP32 clock).  Outputs go to
``tests/golden/*.npz``; the committed fixtures are what the tests read.
"""

from __future__ import annotations

import argparse
import os
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _profiles(ref, pml_cells, dt, resolution, is_3d):
    """Reference CPML profile sampler with resolved sigma/alpha maxima."""
    bc = ref.boundary_compile
    spec = ref.boundaries.PML(formulation="cpml")
    spec = spec.updated_copy(thickness=pml_cells * resolution)
    comp = bc._AbsorberCompiler(spec, cell_thickness=pml_cells)
    fields = types.SimpleNamespace(permittivity=np.zeros((2, 2, 2) if is_3d else (2, 2)))
    sigma_max, alpha_max = comp._resolved_profile_params(fields, resolution, dt)
    spec = spec.updated_copy(sigma_max=sigma_max, alpha_max=alpha_max)
    return bc._AbsorberCompiler(spec, cell_thickness=pml_cells), sigma_max, alpha_max


_H3 = (("Hx", "y"), ("Hx", "z"), ("Hy", "z"), ("Hy", "x"), ("Hz", "x"), ("Hz", "y"))
_E3 = (("Ex", "y"), ("Ex", "z"), ("Ey", "z"), ("Ey", "x"), ("Ez", "x"), ("Ez", "y"))
_AX = {"z": 0, "y": 1, "x": 2}
_FACES = {"z": ("front", "back"), "y": ("bottom", "top"), "x": ("left", "right")}


def _terms_3d(ref, grid, dt, resolution, pml_cells, edges):
    comp, _, _ = _profiles(ref, pml_cells, dt, resolution, True)
    shapes = {c: ref.lattice.component_shape_3d(c, grid) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    out = []
    for specs in (_H3, _E3):
        terms = []
        for i, (c, axis_name) in enumerate(specs):
            axis = _AX[axis_name]
            off = ref.lattice.component_axis_offsets_3d(c)[axis_name]
            kind = "E" if off == 0.0 else "H"
            lo, hi = _FACES[axis_name]
            s, k, a = comp._compute_fdtdx_staggered_profile_1d(
                shapes[c][axis], resolution, lo in edges, hi in edges,
                sample_kind=kind, domain_cells=grid[axis],
            )
            bshape = [1, 1, 1]
            bshape[axis] = shapes[c][axis]
            terms.append(ref.kernels.compile_cpml_term(
                component=c, axis=axis, sign=1.0 if i % 2 == 0 else -1.0,
                sigma=np.reshape(s, bshape), kappa=np.reshape(k, bshape), alpha=np.reshape(a, bshape),
                dt=dt, full_shape=shapes[c],
            ))
        out.append(terms)
    return out[0], out[1], shapes


def _term_arrays(prefix, terms):
    data = {}
    for i, t in enumerate(terms):
        data[f"{prefix}{i}_a"] = np.asarray(t.a).reshape(-1)
        data[f"{prefix}{i}_b"] = np.asarray(t.b).reshape(-1)
        data[f"{prefix}{i}_k"] = np.asarray(t.inv_kappa).reshape(-1)
        data[f"{prefix}{i}_slab"] = np.asarray([t.axis, t.slab.low, t.slab.high, int(t.sign)], np.int32)
    return data


def gen_coefficients(ref):
    sigma = np.asarray([0.0, 0.2, 1.3, 2.1], dtype=np.float32)
    kappa = np.asarray([1.0, 1.0, 2.0, 4.0], dtype=np.float32)
    alpha = np.asarray([0.0, 0.03, 0.02, 0.0], dtype=np.float32)
    dt = 4e-13
    a, b, k = ref.kernels.cpml_coefficients(sigma, kappa, alpha, np.float32(dt))
    data = dict(sigma=sigma, kappa=kappa, alpha=alpha, dt=np.float64(dt),
                a=np.asarray(a), b=np.asarray(b), k=np.asarray(k))
    # Staggered profiles (E and H samples) for a 12-cell default PML.
    res, dt3 = 20e-9, 0.99 * 20e-9 / (299792458.0 * np.sqrt(3.0))
    comp, smax, amax = _profiles(ref, 12, dt3, res, True)
    for kind, n in (("E", 41), ("H", 40)):
        s, kk, al = comp._compute_fdtdx_staggered_profile_1d(n, res, True, True, sample_kind=kind, domain_cells=40)
        data[f"prof{kind}_sigma"], data[f"prof{kind}_kappa"], data[f"prof{kind}_alpha"] = map(np.asarray, (s, kk, al))
        s, kk, al = comp._compute_fdtdx_staggered_profile_1d(n, res, False, True, sample_kind=kind, domain_cells=40)
        data[f"prof{kind}hi_sigma"], data[f"prof{kind}hi_kappa"], data[f"prof{kind}hi_alpha"] = map(np.asarray, (s, kk, al))
    data.update(prof_sigma_max=np.float64(smax), prof_alpha_max=np.float64(amax), prof_dt=np.float64(dt3),
                prof_res=np.float64(res))
    # Known-answer packed recurrence (tests/kernels/test_maxwell_operators.py:132-175 inputs).
    term = ref.kernels.compile_cpml_term(
        component="Ez", axis=0, sign=-1.0,
        sigma=np.asarray([0.8, 0.0, 0.0, 1.1], np.float32), kappa=np.asarray([1.7, 1.0, 1.0, 2.2], np.float32),
        alpha=np.asarray([0.04, 0.0, 0.0, 0.02], np.float32), dt=np.float32(2e-13), full_shape=(4,),
    )
    deriv = np.asarray([1.0, -2.0, 3.0, -4.0], np.float32)
    corrected, psi = ref.kernels.correct_cpml_term(ref.jnp.asarray(deriv), ref.jnp.zeros(term.slab.shape, dtype=np.float32), term)
    data.update(kat_deriv=deriv, kat_corrected=np.asarray(corrected), kat_psi=np.asarray(psi),
                kat_slab=np.asarray([term.slab.low, term.slab.high], np.int32))
    return data


def gen_materials(ref):
    rng = np.random.default_rng(1234)
    vox = rng.choice(np.asarray([2.085, 12.11, 1.0, 4.0], np.float32), size=(5, 6, 7)).astype(np.float32)
    data = {"voxels": vox}
    for c in ("Ex", "Ey", "Ez"):
        data[f"eps_{c}"] = np.asarray(ref.lattice.sample_voxel_grid_at_e_component_3d_centered(vox, c))
    vox2 = rng.choice(np.asarray([2.085, 12.11], np.float32), size=(6, 7)).astype(np.float32)
    data["voxels2d"] = vox2
    for pol, comps in (("tm", ("Ez", "Hx", "Hy")), ("te", ("Ex", "Ey", "Hz"))):
        for c in comps:
            data[f"site2d_{pol}_{c}"] = np.asarray(ref.lattice.sample_voxel_grid_at_component_2d(vox2, c, "xy", pol))
    # PEC masks for a mixed wall set.
    grid = (4, 5, 6)
    shapes = {c: ref.lattice.component_shape_3d(c, grid) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    pec = ref.boundaries.PEC(edges=("front", "top", "left"))
    masks = ref.boundary_compile.compile_metallic_masks(shapes, grid, (pec,))
    for c, m in masks.items():
        data[f"mask_{c}"] = np.asarray(m)
    dt = 1e-17
    sig_m = np.float32(0.0)
    dec, src = ref.kernels.precompute_h_update_coefficients(ref.jnp.asarray(sig_m), dt)
    data["h2d_decay"], data["h2d_source"], data["h2d_dt"] = np.asarray(dec), np.asarray(src), np.float64(dt)
    eps2 = np.asarray(ref.lattice.sample_voxel_grid_at_component_2d(vox2, "Ez", "xy", "tm"))
    dec, src = ref.kernels.precompute_e_update_coefficients(
        shape=eps2.shape, conductivity=ref.jnp.asarray(np.float32(0.0)), permittivity=ref.jnp.asarray(eps2),
        dt=dt, region=(slice(None), slice(None)))
    data["e2d_decay"], data["e2d_source"] = np.asarray(dec), np.asarray(src)
    return data


def _random_fields(rng, shapes, scale=1.0):
    return {c: (rng.standard_normal(shapes[c]) * scale).astype(np.float32) for c in shapes}


def gen_update3d(ref):
    rng = np.random.default_rng(20260724)
    grid = (9, 10, 11)
    res = 20e-9
    dt = 0.99 * res / (299792458.0 * np.sqrt(3.0))
    edges = {"left", "right", "top", "bottom", "front", "back"}
    h_terms, e_terms, shapes = _terms_3d(ref, grid, dt, res, 3, edges)
    fields = _random_fields(rng, shapes)
    fields.update({c: fields[c] * np.float32(1.0 / 376.73) for c in ("Hx", "Hy", "Hz")})
    psi_h = [rng.standard_normal(tuple(t.slab.shape)).astype(np.float32) * np.float32(1e-3) for t in h_terms]
    psi_e = [rng.standard_normal(tuple(t.slab.shape)).astype(np.float32) * np.float32(1e-1) for t in e_terms]
    vox = rng.choice(np.asarray([2.085, 12.11], np.float32), size=grid).astype(np.float32)
    eps = [np.asarray(ref.lattice.sample_voxel_grid_at_e_component_3d_centered(vox, c)) for c in ("Ex", "Ey", "Ez")]
    zero = ref.jnp.asarray(np.float32(0.0))
    jf = {c: ref.jnp.asarray(v) for c, v in fields.items()}
    dt_s = ref.jnp.asarray(dt, dtype=np.float32)
    data = {f"in_{c}": v for c, v in fields.items()}
    data.update({f"in_psi_h{i}": p for i, p in enumerate(psi_h)})
    data.update({f"in_psi_e{i}": p for i, p in enumerate(psi_e)})
    data.update(voxels=vox, dt=np.float64(dt), res=np.float64(res), grid=np.asarray(grid))
    data.update(_term_arrays("h", h_terms))
    data.update(_term_arrays("e", e_terms))
    hx, hy, hz, ph = ref.kernels.cpml_update_h_from_e_3d(
        jf["Ex"], jf["Ey"], jf["Ez"], jf["Hx"], jf["Hy"], jf["Hz"], res,
        terms=h_terms, psi_terms=[ref.jnp.asarray(p) for p in psi_h], dt=dt_s,
        magnetic_conductivities=(zero, zero, zero))
    data.update(cpml_Hx=np.asarray(hx), cpml_Hy=np.asarray(hy), cpml_Hz=np.asarray(hz))
    data.update({f"cpml_psi_h{i}": np.asarray(p) for i, p in enumerate(ph)})
    for tag, metallic in (("open", frozenset()), ("pec", frozenset({"back", "bottom", "right"}))):
        ex, ey, ez, pe = ref.kernels.cpml_update_e_from_h_3d(
            jf["Hx"], jf["Hy"], jf["Hz"], jf["Ex"], jf["Ey"], jf["Ez"], res,
            terms=e_terms, psi_terms=[ref.jnp.asarray(p) for p in psi_e], metallic_edges=metallic, dt=dt_s,
            conductivities=(zero, zero, zero),
            inverse_permittivities=tuple(ref.jnp.reciprocal(ref.jnp.asarray(e)) for e in eps))
        data.update({f"cpml_{tag}_Ex": np.asarray(ex), f"cpml_{tag}_Ey": np.asarray(ey), f"cpml_{tag}_Ez": np.asarray(ez)})
        data.update({f"cpml_{tag}_psi_e{i}": np.asarray(p) for i, p in enumerate(pe)})
    # Plain Yee (no CPML) with PEC ghosts.
    metallic = frozenset({"front", "top", "left"})
    hx, hy, hz = ref.kernels.fused_update_h_lossy_3d_material(
        jf["Ex"], jf["Ey"], jf["Ez"], jf["Hx"], jf["Hy"], jf["Hz"], zero, zero, zero, dt_s, res)
    views = ref.lattice.build_h_boundary_views_for_e_3d(jf["Hx"], jf["Hy"], jf["Hz"], metallic)
    inv = tuple(ref.jnp.reciprocal(ref.jnp.asarray(e)) for e in eps)
    ex, ey, ez = ref.kernels.fused_update_e_lossy_3d_material(
        jf["Hx"], jf["Hy"], jf["Hz"], jf["Ex"], jf["Ey"], jf["Ez"],
        zero, inv[0], zero, inv[1], zero, inv[2], dt_s, res, boundary_views=views)
    data.update(yee_Hx=np.asarray(hx), yee_Hy=np.asarray(hy), yee_Hz=np.asarray(hz),
                yee_Ex=np.asarray(ex), yee_Ey=np.asarray(ey), yee_Ez=np.asarray(ez))
    return data


def _terms_2d(ref, grid, dt, res, pml_cells, pol):
    comp, _, _ = _profiles(ref, pml_cells, dt, res, False)
    ny, nx = grid
    spec = {
        "tm": ((("Hx", 0, 1.0, "H"), ("Hy", 1, -1.0, "H")), (("Ez", 1, 1.0, "E"), ("Ez", 0, -1.0, "E"))),
        "te": ((("Hz", 1, 1.0, "H"), ("Hz", 0, -1.0, "H")), (("Ex", 0, 1.0, "E"), ("Ey", 1, -1.0, "E"))),
    }[pol]
    out = []
    for group in spec:
        terms = []
        for c, axis, sign, kind in group:
            shape = ref.lattice.component_shape_2d(c, grid, "xy", pol)
            cells = grid[axis]
            s, k, a = comp._compute_fdtdx_staggered_profile_1d(shape[axis], res, True, True, sample_kind=kind, domain_cells=cells)
            bshape = [1, 1]
            bshape[axis] = shape[axis]
            terms.append(ref.kernels.compile_cpml_term(
                component=c, axis=axis, sign=sign, sigma=np.reshape(s, bshape), kappa=np.reshape(k, bshape),
                alpha=np.reshape(a, bshape), dt=dt, full_shape=shape))
        out.append(terms)
    return out


def gen_update2d(ref):
    rng = np.random.default_rng(77)
    grid = (13, 15)
    res = 20e-9
    dt = 0.7 * res / (299792458.0 * np.sqrt(2.0))
    data = {"dt": np.float64(dt), "res": np.float64(res), "grid": np.asarray(grid)}
    vox = rng.choice(np.asarray([2.085, 12.11], np.float32), size=grid).astype(np.float32)
    data["voxels"] = vox
    for pol in ("tm", "te"):
        h_terms, e_terms = _terms_2d(ref, grid, dt, res, 3, pol)
        data.update(_term_arrays(f"{pol}h", h_terms))
        data.update(_term_arrays(f"{pol}e", e_terms))
        comps = ("Ez", "Hx", "Hy") if pol == "tm" else ("Ex", "Ey", "Hz")
        f = {c: rng.standard_normal(ref.lattice.component_shape_2d(c, grid, "xy", pol)).astype(np.float32) for c in comps}
        psi_h = [rng.standard_normal(tuple(t.slab.shape)).astype(np.float32) * np.float32(1e-2) for t in h_terms]
        psi_e = [rng.standard_normal(tuple(t.slab.shape)).astype(np.float32) * np.float32(1e-2) for t in e_terms]
        data.update({f"{pol}_in_{c}": v for c, v in f.items()})
        data.update({f"{pol}_in_psi_h{i}": p for i, p in enumerate(psi_h)})
        data.update({f"{pol}_in_psi_e{i}": p for i, p in enumerate(psi_e)})
        jf = {c: ref.jnp.asarray(v) for c, v in f.items()}
        metallic = frozenset({"left", "top"})
        if pol == "tm":
            c0, c1, ph = ref.kernels.tm_xy_cpml_curl_e_to_h_2d(jf["Ez"], res, terms=h_terms, psi_h_terms=[ref.jnp.asarray(p) for p in psi_h])
            ce, pe = ref.kernels.tm_xy_cpml_curl_h_to_e_2d(jf["Hx"], jf["Hy"], res, jf["Ez"].shape, metallic,
                                                          terms=e_terms, psi_e_terms=[ref.jnp.asarray(p) for p in psi_e])
            data.update({f"{pol}_curl_h0": np.asarray(c0), f"{pol}_curl_h1": np.asarray(c1), f"{pol}_curl_e": np.asarray(ce)})
            plain = ref.kernels.tm_xy_curl_h_to_e_2d(jf["Hx"], jf["Hy"], res, jf["Ez"].shape, metallic)
            data[f"{pol}_plain_curl_e"] = np.asarray(plain)
        else:
            ch, ph = ref.kernels.te_xy_cpml_curl_e_to_h_2d(jf["Ex"], jf["Ey"], res, terms=h_terms, psi_h_terms=[ref.jnp.asarray(p) for p in psi_h])
            (ce0, ce1), pe = ref.kernels.te_xy_cpml_curl_h_to_e_2d(jf["Hz"], res, metallic, terms=e_terms,
                                                                  psi_e_terms=[ref.jnp.asarray(p) for p in psi_e])
            data.update({f"{pol}_curl_h": np.asarray(ch), f"{pol}_curl_e0": np.asarray(ce0), f"{pol}_curl_e1": np.asarray(ce1)})
            p0, p1 = ref.kernels.te_xy_curl_h_to_e_2d(jf["Hz"], res, jf["Ex"].shape, jf["Ey"].shape, metallic)
            data[f"{pol}_plain_curl_e0"], data[f"{pol}_plain_curl_e1"] = np.asarray(p0), np.asarray(p1)
        data.update({f"{pol}_psi_h{i}": np.asarray(p) for i, p in enumerate(ph)})
        data.update({f"{pol}_psi_e{i}": np.asarray(p) for i, p in enumerate(pe)})
    return data


def gen_pulse(ref):
    dt = 0.99 * 20e-9 / (299792458.0 * np.sqrt(3.0))
    f0 = 299792458.0 / 1.55e-6
    times = (np.arange(200, dtype=np.float64) + 0.5) * dt
    pulse = ref.time.GaussianPulse(freq0=f0, fwidth=0.2 * f0, offset=0.5)
    sig, quad = pulse.sample(times)
    pulse2 = ref.time.GaussianPulse(freq0=f0, fwidth=0.1 * f0, amplitude=2.0, offset=4.0, remove_dc_component=False)
    sig2, _ = pulse2.sample(times)
    return dict(times=times, f0=np.float64(f0), signal=np.asarray(sig), quadrature=np.asarray(quad), signal2=np.asarray(sig2))


def _monitor_ns(ref, freqs, idx, w, mask, t0, t1, interval, window, norm, unit, voff, woff, npt):
    return types.SimpleNamespace(
        freq_hz=np.asarray(freqs, np.float32), dft_t_start=t0, dft_t_end=t1, dft_window_code=window,
        dft_normalization_code=norm, dft_record_interval=interval, dft_length_unit=unit,
        dft_flat_idx=[ref.jnp.asarray(i) for i in idx], dft_weights=[ref.jnp.asarray(x) for x in w],
        dft_component_mask=ref.jnp.asarray(mask), freq_count=len(freqs), dft_point_count=npt,
        dft_value_offset=voff, dft_weight_offset=woff,
    )


def gen_dft(ref):
    rng = np.random.default_rng(5)
    grid = (6, 7, 8)
    res = 20e-9
    shapes = {c: ref.lattice.component_shape_3d(c, grid) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    fields = {c: rng.standard_normal(shapes[c]).astype(np.float32) for c in shapes}
    coords0 = (np.arange(4) + 1.3) * res  # z
    coords1 = (np.arange(5) + 0.7) * res  # y
    idx, w = [], []
    for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        fi, fw = ref.lattice._component_plane_plan_3d(
            c, normal_axis="x", plane_position=3.25 * res, coordinates=(coords0, coords1),
            resolution=res, grid_shape=grid, field_shape=shapes[c])
        idx.append(np.asarray(fi))
        w.append(np.asarray(fw))
    # Pad to a common K (the CUDA arena uses one neighbour count).
    k = max(a.shape[1] for a in idx)
    idx_p = [np.pad(a, ((0, 0), (0, k - a.shape[1]))) for a in idx]
    w_p = [np.pad(a, ((0, 0), (0, k - a.shape[1]))) for a in w]
    npt = idx[0].shape[0]
    freqs = np.asarray([1.8e14, 1.93e14, 2.05e14], np.float32)
    mask = np.asarray([0, 1, 1, 0, 1, 1], np.float32)
    dt = 0.99 * res / (299792458.0 * np.sqrt(3.0))
    nf = len(freqs)
    re = ref.jnp.asarray(rng.standard_normal(6 * nf * npt).astype(np.float32))
    im = ref.jnp.asarray(rng.standard_normal(6 * nf * npt).astype(np.float32))
    ww = ref.jnp.asarray(np.zeros(nf, np.float32))
    data = {f"f_{c}": v for c, v in fields.items()}
    data.update({f"idx_{i}": a for i, a in enumerate(idx_p)})
    data.update({f"w_{i}": a for i, a in enumerate(w_p)})
    data.update(freqs=freqs, mask=mask, dt=np.float64(dt), re0=np.asarray(re), im0=np.asarray(im), grid=np.asarray(grid))
    fa = tuple(ref.jnp.asarray(fields[c]) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"))
    cases = (("plain", 0, 0, 0.0, float("inf"), 1, 37.0 * dt),
             ("hann", 1, 1, 5.0 * dt, 120.0 * dt, 1, 37.0 * dt))
    for tag, window, norm, t0, t1, interval, t_phys in cases:
        mon = _monitor_ns(ref, freqs, idx_p, w_p, mask, t0, t1, interval, window, norm, 1e-6, 0, 0, npt)
        tp = np.float32(t_phys)
        gate = ref.observe.monitor_dft_should_accumulate(True, 36, tp, t0, t1, interval)
        r, i_, wsum = ref.observe._accumulate_dft(mon, (re, im, ww), fa, tp, ref.jnp.asarray(dt, dtype=np.float32))
        data.update({f"{tag}_re": np.asarray(r), f"{tag}_im": np.asarray(i_), f"{tag}_w": np.asarray(wsum),
                     f"{tag}_gate": np.asarray(bool(gate)), f"{tag}_t": np.float32(tp),
                     f"{tag}_cfg": np.asarray([window, norm, t0, t1, interval], np.float64)})
    return data


def _apply_slab(arr, start, coeff, amp):
    sl = tuple(slice(s, s + n) for s, n in zip(start, coeff.shape))
    out = np.array(arr, copy=True)
    out[sl] = out[sl] + (coeff * np.float32(amp)).astype(np.float32)
    return out


def gen_steps3d(ref, nsteps=16):
    """Compose the reference kernels in forward_step order on a small grid."""
    rng = np.random.default_rng(99)
    grid = (10, 11, 12)
    res = 20e-9
    dt = 0.99 * res / (299792458.0 * np.sqrt(3.0))
    edges = {"left", "right", "top", "bottom", "back"}  # CPML faces
    metallic = frozenset({"front"})
    h_terms, e_terms, shapes = _terms_3d(ref, grid, dt, res, 3, edges)
    vox = np.full(grid, 2.085, np.float32)
    vox[3:7, 4:8, 2:9] = 12.11
    eps = [np.asarray(ref.lattice.sample_voxel_grid_at_e_component_3d_centered(vox, c)) for c in ("Ex", "Ey", "Ez")]
    inv = tuple(ref.jnp.reciprocal(ref.jnp.asarray(e)) for e in eps)
    masks = ref.boundary_compile.compile_metallic_masks(shapes, grid, (ref.boundaries.PEC(edges=("front",)),))
    f0 = 299792458.0 / 1.55e-6
    times = (np.arange(nsteps) + 0.5) * dt
    pulse = ref.time.GaussianPulse(freq0=f0, fwidth=0.5 * f0, offset=0.3)
    wave, _ = pulse.sample(times)
    wave = np.asarray(wave)
    src_start = (5, 5, 6)
    src_coeff = np.asarray([[[-dt / (8.8541878128e-12 * 2.085)]]], np.float32)
    hwave = (rng.standard_normal(nsteps) * 1e-3).astype(np.float32)
    h_start, h_coeff = (2, 3, 4), rng.standard_normal((1, 2, 3)).astype(np.float32)
    # DFT: one x-normal plane of Ey/Ez/Hy/Hz.
    coords0 = (np.arange(3) + 3.5) * res
    coords1 = (np.arange(4) + 3.5) * res
    idx, w = [], []
    for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        fi, fw = ref.lattice._component_plane_plan_3d(c, normal_axis="x", plane_position=8.0 * res,
                                                    coordinates=(coords0, coords1), resolution=res,
                                                    grid_shape=grid, field_shape=shapes[c])
        idx.append(np.asarray(fi))
        w.append(np.asarray(fw))
    k = max(a.shape[1] for a in idx)
    idx = [np.pad(a, ((0, 0), (0, k - a.shape[1]))) for a in idx]
    w = [np.pad(a, ((0, 0), (0, k - a.shape[1]))) for a in w]
    npt = idx[0].shape[0]
    freqs = np.asarray([0.9 * f0, f0, 1.1 * f0], np.float32)
    cmask = np.asarray([0, 1, 1, 0, 1, 1], np.float32)
    mon = _monitor_ns(ref, freqs, idx, w, cmask, 0.0, float("inf"), 1, 0, 0, 1e-6, 0, 0, npt)
    re = ref.jnp.zeros(6 * 3 * npt, dtype=np.float32)
    im = ref.jnp.zeros(6 * 3 * npt, dtype=np.float32)
    ws = ref.jnp.zeros(3, dtype=np.float32)
    f = {c: np.zeros(shapes[c], np.float32) for c in shapes}
    psi_h = [ref.jnp.zeros(tuple(t.slab.shape), dtype=np.float32) for t in h_terms]
    psi_e = [ref.jnp.zeros(tuple(t.slab.shape), dtype=np.float32) for t in e_terms]
    zero = ref.jnp.asarray(np.float32(0.0))
    dt_s = ref.jnp.asarray(dt, dtype=np.float32)
    t = np.float32(0.0)
    for step in range(nsteps):
        f["Ey"] = _apply_slab(f["Ey"], src_start, src_coeff, wave[min(step, nsteps - 1)])
        hx, hy, hz, psi_h = ref.kernels.cpml_update_h_from_e_3d(
            ref.jnp.asarray(f["Ex"]), ref.jnp.asarray(f["Ey"]), ref.jnp.asarray(f["Ez"]),
            ref.jnp.asarray(f["Hx"]), ref.jnp.asarray(f["Hy"]), ref.jnp.asarray(f["Hz"]), res,
            terms=h_terms, psi_terms=psi_h, dt=dt_s, magnetic_conductivities=(zero, zero, zero))
        f["Hx"], f["Hy"], f["Hz"] = (np.asarray(v) for v in (hx, hy, hz))
        f["Hz"] = _apply_slab(f["Hz"], h_start, h_coeff, hwave[step])
        for c in ("Hx", "Hy", "Hz"):
            f[c] = np.asarray(ref.kernels.apply_zero_mask(ref.jnp.asarray(f[c]), masks[c]))
        ex, ey, ez, psi_e = ref.kernels.cpml_update_e_from_h_3d(
            ref.jnp.asarray(f["Hx"]), ref.jnp.asarray(f["Hy"]), ref.jnp.asarray(f["Hz"]),
            ref.jnp.asarray(f["Ex"]), ref.jnp.asarray(f["Ey"]), ref.jnp.asarray(f["Ez"]), res,
            terms=e_terms, psi_terms=psi_e, metallic_edges=metallic, dt=dt_s,
            conductivities=(zero, zero, zero), inverse_permittivities=inv)
        f["Ex"], f["Ey"], f["Ez"] = (np.asarray(v) for v in (ex, ey, ez))
        for c in ("Ex", "Ey", "Ez"):
            f[c] = np.asarray(ref.kernels.apply_zero_mask(ref.jnp.asarray(f[c]), masks[c]))
        t_phys = np.float32(t + np.float32(dt))
        fa = tuple(ref.jnp.asarray(f[c]) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"))
        if bool(ref.observe.monitor_dft_should_accumulate(True, step, t_phys, 0.0, float("inf"), 1)):
            re, im, ws = ref.observe._accumulate_dft(mon, (re, im, ws), fa, t_phys, dt_s)
        t = t_phys
    data = {f"out_{c}": v for c, v in f.items()}
    data.update({f"out_psi_h{i}": np.asarray(p) for i, p in enumerate(psi_h)})
    data.update({f"out_psi_e{i}": np.asarray(p) for i, p in enumerate(psi_e)})
    data.update(dft_re=np.asarray(re), dft_im=np.asarray(im), dft_w=np.asarray(ws), t=np.float32(t))
    data.update(voxels=vox, wave=wave, hwave=hwave, h_coeff=h_coeff, src_coeff=src_coeff,
                freqs=freqs, cmask=cmask, dt=np.float64(dt), res=np.float64(res), nsteps=np.int32(nsteps),
                grid=np.asarray(grid))
    data.update({f"idx_{i}": a for i, a in enumerate(idx)})
    data.update({f"w_{i}": a for i, a in enumerate(w)})
    data.update(_term_arrays("h", h_terms))
    data.update(_term_arrays("e", e_terms))
    return data


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("BEAMZ_REFERENCE_ROOT"),
                        help="root of the beamz source tree (or set BEAMZ_REFERENCE_ROOT)")
    args = parser.parse_args()
    if not args.reference:
        parser.error("--reference (or BEAMZ_REFERENCE_ROOT) is required")
    os.environ["BEAMZ_REFERENCE_ROOT"] = args.reference
    from ._refload import load_reference

    ref = load_reference()
    for name, fn in (
        ("coefficients", gen_coefficients),
        ("materials", gen_materials),
        ("update3d", gen_update3d),
        ("update2d", gen_update2d),
        ("pulse", gen_pulse),
        ("dft", gen_dft),
        ("steps3d", gen_steps3d),
    ):
        data = fn(ref)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"wrote {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
