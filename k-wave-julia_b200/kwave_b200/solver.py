"""``kspace_first_order`` on the GPU through libkwb, with the reference's signature and output.

``kspace_first_order(kgrid, medium, source, sensor; ...)`` (KWave.jl/src/solver/
first_order.jl:92-111, 287-306, 505-524) is restated as: validate and normalise the arguments
exactly where the reference does, smooth p0 on the host in FP64 (first_order_steps.jl:70-72,
109-111, 157-159), build one ``kwb_problem`` and call ``kwb_solve``; then apply the reference's
post-loop host filters (first_order_steps.jl:836-910) and return a ``SimulationOutput``.

``kspace_first_order_as`` (solver/axisymmetric.jl:26-227) and ``pstd_elastic_2d`` /
``pstd_elastic_3d`` (solver/elastic.jl:133-588) go through the same ``kwb_problem`` with its
axisymmetric or elastic fields set; the elastic solvers return the recorded data without the
post-loop filters, as the reference does.

Errors the reference raises are raised here with the same meaning: an unset time array, an
invalid record field, signals with too few rows (BoundsError), ``:I_avg``/``:I_max`` with
``data_cast=Float32`` (MethodError in ``_acoustic_intensity``), array ``alpha_coeff``.
"""

from __future__ import annotations

import ctypes as C
import threading
import warnings
from typing import Optional

import numpy as np

from . import _lib
from ._lib import KWaveB200Error, check
from .core import (ElasticMedium, ElasticSource, KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource,
                   SimulationOutput, SourceMode, smooth, validate_record_fields)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _ptr_d(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ptr_i(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _flat(a, shape) -> np.ndarray:
    """A grid-shaped array as a row-major (C-order) FP64 buffer, without a copy when it already
    is one; the library reorders it to the reference's column-major layout on the device
    (kwb_problem.row_major = 1).  A flat vector of the grid's size is read as column-major
    (Julia linear order), as the reference would."""
    arr = np.asarray(a, dtype=np.float64)
    if arr.shape != tuple(shape):
        if arr.size == int(np.prod(shape)) and arr.ndim == 1:
            return _f64(arr.reshape(tuple(shape), order="F"))
        raise ValueError(f"array of shape {arr.shape} does not match the grid {tuple(shape)}")
    return _f64(arr)


def _findall(mask, shape) -> np.ndarray:
    """findall(mask) - 1: sorted 0-based column-major linear indices of the True entries."""
    m = np.asarray(mask, dtype=bool)
    if m.shape != tuple(shape):
        raise ValueError(f"mask of shape {m.shape} does not match the grid {tuple(shape)}")
    if m.ndim > 1 and 4 * int(np.count_nonzero(m)) <= m.size:
        # sparse: row-major flat indices of the points (one scan of the mask), mapped to
        # column-major linear indices and sorted
        k = np.flatnonzero(m.reshape(-1))
        lin = np.zeros(k.size, dtype=np.int64)
        col_stride = 1
        for ax in range(m.ndim):
            c, k = np.divmod(k, int(np.prod(m.shape[ax + 1:], dtype=np.int64)))
            lin += c * col_stride
            col_stride *= m.shape[ax]
        lin.sort()
        return lin
    return np.ascontiguousarray(np.flatnonzero(m.ravel(order="F")).astype(np.int64))


def _signal(sig) -> np.ndarray:
    """A vector signal indexes as an n x 1 matrix (size(v, 2) == 1 in Julia)."""
    s = np.asarray(sig, dtype=np.float64)
    if s.ndim == 1:
        s = s.reshape(-1, 1)
    if s.ndim != 2:
        raise ValueError("source signals must be vectors or (n_points x n_cols) matrices")
    return np.ascontiguousarray(s.ravel(order="F")), s.shape[0], s.shape[1]


class Context:
    """A libkwb context bound to one CUDA device (use from one thread at a time)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load_library()
        h = C.c_void_p()
        rc = self.lib.kwb_context_create(device, C.byref(h))
        if rc != _lib.KWB_OK:
            msg = self.lib.kwb_last_error(None)
            raise KWaveB200Error(rc, msg.decode() if msg else "context creation failed")
        self.handle = h
        self.device = device
        self.lock = threading.Lock()

    def close(self):
        if self.handle:
            self.lib.kwb_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None
_default_lock = threading.Lock()


def default_context() -> Context:
    global _default_ctx
    with _default_lock:
        if _default_ctx is None:
            _default_ctx = Context(0)
        return _default_ctx


class _Built:
    """A kwb_problem plus every host array it points into (kept alive for the call)."""

    def __init__(self):
        self.keep = []
        self.problem = _lib.Problem()
        self.groups_py = []  # (record list, n_rows) per group
        self.callback = None

    def arr(self, a):
        self.keep.append(a)
        return a


def _warn_fp32(data_cast):
    """The reference's default data_cast=Float64 asks for an FP64 solve; this path steps in FP32."""
    if np.dtype(data_cast) == np.float64:
        warnings.warn("kwave_b200 steps fields and FFTs in FP32 on the GPU; outputs stay float64 and agree "
                      "with the reference's Float64 solve to about 1e-5 relative L2 (data_cast=float64 is "
                      "not an FP64 GPU solve)", RuntimeWarning, stacklevel=3)


def build_problem(kgrid: KWaveGrid, medium: KWaveMedium, source: KWaveSource, sensor: KWaveSensor,
                  pml_size=20, pml_alpha=2.0, smooth_p0: bool = True, data_cast=np.float64,
                  progress_callback=None, extra_sensors=(), axisymmetric: bool = False,
                  elastic: bool = False) -> _Built:
    """Normalise the reference's arguments into a kwb_problem (first_order.jl:311-441, 529-669).

    An ``ElasticMedium`` (or ``elastic=True``) selects the stress-velocity solver
    (solver/elastic.jl:133-588) with an ``ElasticSource``: p0 is not smoothed and time-reversal
    data is not used.

    ``extra_sensors`` (not in the reference API) adds further sensor groups -- (mask, record)
    pairs given as ``KWaveSensor`` or dicts -- so one solve can record different fields on
    different masks; their outputs come back in ``SimulationOutput.extra``.
    """
    if kgrid.Nt == 0 or kgrid.dt == 0:
        raise RuntimeError("Time array not set. Call make_time!(kgrid, sound_speed) before running.")
    validate_record_fields(sensor)
    D = kgrid.ndim
    shape = kgrid.N
    nvox = int(np.prod(shape))
    b = _Built()
    P = b.problem
    P.ndim = D
    for a in range(3):
        P.N[a] = shape[a] if a < D else 1
        P.d[a] = kgrid.d[a] if a < D else 1.0
    P.dt = float(kgrid.dt)
    P.Nt = int(kgrid.Nt)
    P.row_major = 1  # grid arrays go over as NumPy (row-major) buffers; see _flat
    P.axisymmetric = 1 if axisymmetric else 0
    elastic = elastic or isinstance(medium, ElasticMedium)
    P.elastic = 1 if elastic else 0
    if elastic and D not in (2, 3):
        raise TypeError("the elastic solver takes a 2D or 3D grid")
    if D == 1:
        if isinstance(pml_size, (tuple, list)) or isinstance(pml_alpha, (tuple, list)):
            raise TypeError("the 1D solver takes scalar pml_size and pml_alpha")
    psz = tuple(pml_size) if isinstance(pml_size, (tuple, list)) else (pml_size,) * D
    pal = tuple(pml_alpha) if isinstance(pml_alpha, (tuple, list)) else (pml_alpha,) * D
    if len(psz) != D or len(pal) != D:
        raise TypeError("pml_size / pml_alpha tuples must have one entry per dimension")
    for a in range(D):
        P.pml_size[a] = int(psz[a])
        P.pml_alpha[a] = float(pal[a])

    def field(v, name, optional=False):
        f = _lib.Field()
        if v is None:
            if not optional:
                raise TypeError(f"{name} is required")
            f.count = 0
            return f
        arr = b.arr(_f64([float(v)]) if np.ndim(v) == 0 else _flat(v, shape))
        f.data = _ptr_d(arr)
        f.count = arr.size
        return f

    if elastic:
        _elastic_medium(P, medium, field, D)
    else:
        P.c0 = field(medium.sound_speed, "sound_speed")
        P.rho0 = field(medium.density if medium.density is not None else 1.0, "density")
        P.BonA = field(medium.BonA, "BonA", optional=True)
    if elastic:
        pass
    elif medium.is_lossless():
        P.alpha_mode = _lib.NO_ABSORPTION
    else:
        if np.ndim(medium.alpha_coeff) != 0:
            raise TypeError("array alpha_coeff is not supported by the reference solver "
                            "(T(absorb_tau) on an array, first_order.jl:369)")
        if medium.alpha_power is None:
            raise TypeError("alpha_power must be set when alpha_coeff is set (db2neper(x, nothing))")
        modes = {"no_absorption": _lib.NO_ABSORPTION, "no_dispersion": _lib.NO_DISPERSION,
                 "stokes": _lib.STOKES}
        if medium.alpha_mode not in modes:
            raise ValueError(f"unknown alpha_mode {medium.alpha_mode}")
        P.alpha_mode = modes[medium.alpha_mode]
        P.alpha_coeff = float(medium.alpha_coeff)
        P.alpha_power = float(medium.alpha_power)

    # the axisymmetric and elastic solvers ignore time-reversal data
    tr = sensor.is_time_reversal() and not axisymmetric and not elastic
    if source.p0 is not None and not tr:
        p0 = np.asarray(source.p0, dtype=np.float64)
        if p0.shape != tuple(shape):
            raise ValueError(f"p0 of shape {p0.shape} does not match the grid {tuple(shape)}")
        do_smooth = not elastic and smooth_p0 and ((D == 1 and shape[0] > 4) or (D > 1 and all(n > 1 for n in shape)))
        if do_smooth:
            p0 = smooth(p0, restore_max=True)
        arr = b.arr(_flat(p0, shape))
        P.p0.data = _ptr_d(arr)
        P.p0.count = nvox

    if elastic and source.has_stress_source():
        idx = b.arr(_findall(source.s_mask, shape))
        P.s_index = _ptr_i(idx)
        P.n_s_index = idx.size
        P.s_mode = int(SourceMode(source.s_mode))
        comps = (source.sxx, source.syy, source.szz, source.sxy, source.sxz, source.syz)
        for k, comp in enumerate(comps):
            if comp is None or (D == 2 and k in (2, 4, 5)):  # the 2D solver reads sxx, syy, sxy
                continue
            sig, rows, cols = _signal(comp)
            b.arr(sig)
            if rows < idx.size and idx.size > 0:
                raise IndexError(f"BoundsError: stress signal {k} has {rows} rows for {idx.size} s_mask points")
            P.s_signal[k].data = _ptr_d(sig)
            P.s_signal[k].n_rows = rows
            P.s_signal[k].n_cols = cols
    if not elastic and source.has_pressure_source():
        idx = b.arr(_findall(source.p_mask, shape))
        sig, rows, cols = _signal(source.p)
        b.arr(sig)
        if rows < idx.size:
            raise IndexError(f"BoundsError: source.p has {rows} rows for {idx.size} p_mask points")
        P.p_index = _ptr_i(idx)
        P.n_p_index = idx.size
        P.p_mode = int(SourceMode(source.p_mode))
        P.p_signal.data = _ptr_d(sig)
        P.p_signal.n_rows = rows
        P.p_signal.n_cols = cols
    if source.has_velocity_source():
        idx = b.arr(_findall(source.u_mask, shape))
        P.u_index = _ptr_i(idx)
        P.n_u_index = idx.size
        P.u_mode = int(SourceMode(source.u_mode))
        for a, comp in enumerate((source.ux, source.uy, source.uz)):
            if comp is None or a >= D:
                continue
            sig, rows, cols = _signal(comp)
            b.arr(sig)
            if rows < idx.size and idx.size > 0:
                raise IndexError(f"BoundsError: velocity signal {a} has {rows} rows for {idx.size} u_mask points")
            P.u_signal[a].data = _ptr_d(sig)
            P.u_signal[a].n_rows = rows
            P.u_signal[a].n_cols = cols

    groups = []
    sensors = [sensor] + [s if isinstance(s, KWaveSensor) else KWaveSensor(**s) for s in extra_sensors]
    for gi, sen in enumerate(sensors):
        if sen.mask is None:
            if gi == 0:
                continue
            raise ValueError("extra sensors need a mask")
        validate_record_fields(sen)
        m = np.asarray(sen.mask)
        g = _lib.SensorGroup()
        if m.dtype == bool:
            if m.shape == tuple(shape) and nvox > 0 and m.all():
                g.dense = 1  # every voxel, in linear order: no index list
                g.n_index = nvox
                n_rows = nvox
            else:
                idx = b.arr(_findall(m, shape))
                g.index = _ptr_i(idx)
                g.n_index = idx.size
                n_rows = idx.size
        else:
            g.cartesian = 1
            g.n_index = int(m.shape[1])
            n_rows = int(m.shape[1])
        rec = list(sen.record)
        if ("I_avg" in rec or "I_max" in rec) and np.dtype(data_cast) == np.float32 and n_rows > 0 \
                and m.dtype == bool and not elastic:
            raise TypeError("MethodError: _acoustic_intensity(::Float32, ...) -- the reference records "
                            ":I_avg/:I_max only with data_cast=Float64")
        for f in rec:
            g.record_mask |= 1 << _lib.REC[f]
            g.record_count[_lib.REC[f]] += 1
        if gi == 0 and not elastic and m.dtype == bool:
            # post-loop filters of p (first_order_steps.jl:836-910), applied by the library on the
            # device before read-back; the elastic solvers have none
            if sen.directivity_angle is not None and sen.directivity_size is not None:
                ang = np.asarray(sen.directivity_angle, dtype=np.float64)
                flat = b.arr(np.ascontiguousarray(ang.ravel(order="F")))
                if ang.ndim > 0 and flat.size < n_rows:
                    raise IndexError(f"BoundsError: directivity_angle has {flat.size} entries for {n_rows} sensor points")
                g.directivity_angle = _ptr_d(flat)
                g.n_directivity_angle = 1 if ang.ndim == 0 else flat.size
                g.directivity_size = float(sen.directivity_size)
            if sen.frequency_response is not None:
                fc, bw = sen.frequency_response
                g.has_frequency_response = 1
                g.frequency_center = float(fc)
                g.frequency_bandwidth = float(bw)
        groups.append(g)
        b.groups_py.append((rec, n_rows, bool(g.cartesian)))
    if groups:
        arr = (_lib.SensorGroup * len(groups))(*groups)
        b.keep.append(arr)
        P.groups = arr
        P.n_groups = len(groups)

    if tr:
        data = np.asarray(sensor.time_reversal_boundary_data, dtype=np.float64)
        if data.ndim == 1:
            data = data.reshape(-1, 1)
        flat = b.arr(np.ascontiguousarray(data.ravel(order="F")))
        P.tr.data = _ptr_d(flat)
        P.tr.n_rows = data.shape[0]
        P.tr.n_cols = data.shape[1]

    if progress_callback is not None:
        def _cb(t_index, Nt, p_ptr, user):
            p = np.ctypeslib.as_array(p_ptr, shape=(nvox,)).reshape(shape, order="F").copy()
            progress_callback(int(t_index), int(Nt), p)
        b.callback = _lib.PROGRESS_FN(_cb)
        P.progress = b.callback
    return b


def _elastic_medium(P, medium, field, D):
    """ElasticMedium -> kwb_problem: speeds, density and the Kelvin-Voigt coefficients
    (solver/elastic.jl:164-195)."""
    cp, cs, rho = medium.sound_speed_compression, medium.sound_speed_shear, medium.density
    if np.ndim(rho) == 0 and (np.ndim(cp) != 0 or np.ndim(cs) != 0):
        raise TypeError("MethodError: a scalar density with array wave speeds is evaluated as a matrix "
                        "power (cp^2) by the reference (solver/elastic.jl:169); give the density as an array")
    P.c0 = field(cp, "sound_speed_compression")
    P.cs = field(cs, "sound_speed_shear")
    P.rho0 = field(1000.0 if rho is None else rho, "density")
    y = medium.alpha_power
    used = D == 2 and np.ndim(rho) == 0  # chi enters the 2D homogeneous branch only
    for name in ("alpha_coeff_compression", "alpha_coeff_shear"):
        a = getattr(medium, name)
        if a is not None and used and np.ndim(a) != 0:
            raise TypeError(f"array {name} is not supported (the homogeneous 2D branch scales by it)")
    if y is not None:
        P.alpha_power = float(y)
        if medium.alpha_coeff_compression is not None and used:
            P.alpha_mode = _lib.NO_DISPERSION  # any absorbing mode: the elastic step reads only chi
            P.alpha_coeff = float(medium.alpha_coeff_compression)
        if medium.alpha_coeff_shear is not None and used:
            P.has_alpha_shear = 1
            P.alpha_coeff_shear = float(medium.alpha_coeff_shear)


def _alloc_outputs(ctx: Context, b: _Built, kgrid: KWaveGrid):
    lib = ctx.lib
    ng = b.problem.n_groups
    sizes = (_lib.GroupSizes * max(ng, 1))()
    pf_len = C.c_int64(0)
    check(lib, ctx.handle, lib.kwb_query_outputs(ctx.handle, C.byref(b.problem), sizes, C.byref(pf_len)))
    outs = (_lib.GroupOutputs * max(ng, 1))()
    arrays = []
    for g in range(ng):
        rec, _, _ = b.groups_py[g]
        d = {}
        for f in dict.fromkeys(rec):
            i = _lib.REC[f]
            rows, cols = sizes[g].rows[i], sizes[g].cols[i]
            a = np.zeros(rows * cols, dtype=np.float64)
            outs[g].field[i] = _ptr_d(a)
            d[f] = (a, rows, cols)
        arrays.append(d)
    O = _lib.Outputs()
    O.groups = outs
    pfull = None
    if pf_len.value > 0:
        pfull = np.zeros(pf_len.value, dtype=np.float64)
        O.p_final_full = _ptr_d(pfull)
    return O, outs, arrays, pfull


def _collect(b: _Built, arrays, pfull, sensor: KWaveSensor, kgrid: KWaveGrid, Nt_loop: int):
    dicts = []
    for g, d in enumerate(arrays):
        data = {}
        for f, (a, rows, cols) in d.items():
            data[f] = a.reshape((rows, cols), order="F") if f in _lib.SERIES_FIELDS else a
        dicts.append(data)
    main = dicts[0] if (dicts and sensor.mask is not None) else {}
    extra = dicts[1:] if sensor.mask is not None else dicts
    if pfull is not None:
        main["p_final"] = pfull
    out = SimulationOutput(main)
    out.extra = extra
    return out


def kspace_first_order(kgrid: KWaveGrid, medium: KWaveMedium, source: KWaveSource,
                       sensor: KWaveSensor, *, pml_inside: bool = True, pml_size=20,
                       pml_alpha=2.0, smooth_p0: bool = True, smooth_c0: bool = False,
                       smooth_rho0: bool = False, data_cast=np.float64, save_to_disk=None,
                       plot_sim: bool = False, plot_layout: str = "default", plot_scale="auto",
                       record_movie=None, progress_callback=None, show_progress: bool = True,
                       context: Optional[Context] = None) -> SimulationOutput:
    """Run the fluid k-space simulation on the GPU; same arguments and output as the reference.

    ``pml_inside``, ``smooth_c0``, ``smooth_rho0``, ``plot_*``, ``record_movie`` and
    ``show_progress`` are accepted and ignored, as in the reference solver body.  Fields and
    FFTs are FP32 whatever ``data_cast`` says; ``data_cast`` only selects the reference's error
    behaviour for ``:I_avg``/``:I_max``.
    """
    _warn_fp32(data_cast)
    if save_to_disk is not None:
        raise NotImplementedError("save_to_disk writes an HDF5 input file for the k-Wave C++ binary; "
                                  "HDF5 output is not part of this library")
    ctx = context or default_context()
    b = build_problem(kgrid, medium, source, sensor, pml_size=pml_size, pml_alpha=pml_alpha,
                      smooth_p0=smooth_p0, data_cast=data_cast, progress_callback=progress_callback)
    Nt_loop = b.problem.tr.n_cols if b.problem.tr.data else b.problem.Nt
    with ctx.lock:
        O, outs, arrays, pfull = _alloc_outputs(ctx, b, kgrid)
        check(ctx.lib, ctx.handle, ctx.lib.kwb_solve(ctx.handle, C.byref(b.problem), C.byref(O)))
    if sensor.is_time_reversal():
        kgrid.Nt = int(Nt_loop)  # the reference mutates kgrid.Nt[] (first_order.jl:430-431)
    return _collect(b, arrays, pfull, sensor, kgrid, Nt_loop)


def kspace_first_order_as(kgrid: KWaveGrid, medium: KWaveMedium, source: KWaveSource,
                          sensor: KWaveSensor, *, pml_inside: bool = True, pml_size=20,
                          pml_alpha=2.0, smooth_p0: bool = True, smooth_c0: bool = False,
                          smooth_rho0: bool = False, data_cast=np.float64, plot_sim: bool = False,
                          plot_layout: str = "default", plot_scale="auto", record_movie=None,
                          progress_callback=None, context: Optional[Context] = None) -> SimulationOutput:
    """Axisymmetric solve on a 2D grid, x axial and y radial (``kspace_first_order_as``,
    solver/axisymmetric.jl:26-227): the 2D time step with u_r / r added to the radial divergence.
    Same arguments and output as the reference; like it, time-reversal data on the sensor is not
    used (the sensor records as usual)."""
    if kgrid.ndim != 2:
        raise TypeError("MethodError: kspace_first_order_as takes a KWaveGrid2D (x axial, y radial)")
    ctx = context or default_context()
    b = build_problem(kgrid, medium, source, sensor, pml_size=pml_size, pml_alpha=pml_alpha,
                      smooth_p0=smooth_p0, data_cast=data_cast, progress_callback=progress_callback,
                      axisymmetric=True)
    with ctx.lock:
        O, outs, arrays, pfull = _alloc_outputs(ctx, b, kgrid)
        check(ctx.lib, ctx.handle, ctx.lib.kwb_solve(ctx.handle, C.byref(b.problem), C.byref(O)))
    return _collect(b, arrays, pfull, sensor, kgrid, int(b.problem.Nt))


def _pstd_elastic(kgrid, medium, source, sensor, pml_size, pml_alpha, progress_callback, context):
    ctx = context or default_context()
    b = build_problem(kgrid, medium, source, sensor, pml_size=pml_size, pml_alpha=pml_alpha,
                      progress_callback=progress_callback, elastic=True)
    with ctx.lock:
        O, outs, arrays, pfull = _alloc_outputs(ctx, b, kgrid)
        check(ctx.lib, ctx.handle, ctx.lib.kwb_solve(ctx.handle, C.byref(b.problem), C.byref(O)))
    return _collect(b, arrays, pfull, sensor, kgrid, int(b.problem.Nt))


def pstd_elastic_2d(kgrid: KWaveGrid, medium: ElasticMedium, source: ElasticSource, sensor: KWaveSensor,
                    *, pml_size=20, pml_alpha=2.0, data_cast=np.float64, plot_sim: bool = False,
                    progress_callback=None, context: Optional[Context] = None) -> SimulationOutput:
    """2D elastic stress-velocity PSTD solve on the GPU (``pstd_elastic_2d``,
    solver/elastic.jl:133-366); same arguments and output as the reference.  Fields and FFTs are
    FP32; ``data_cast`` and ``plot_sim`` are accepted and ignored."""
    if kgrid.ndim != 2:
        raise TypeError("MethodError: pstd_elastic_2d takes a KWaveGrid2D")
    return _pstd_elastic(kgrid, medium, source, sensor, pml_size, pml_alpha, progress_callback, context)


def pstd_elastic_3d(kgrid: KWaveGrid, medium: ElasticMedium, source: ElasticSource, sensor: KWaveSensor,
                    *, pml_size=10, pml_alpha=2.0, data_cast=np.float64, plot_sim: bool = False,
                    progress_callback=None, context: Optional[Context] = None) -> SimulationOutput:
    """3D elastic stress-velocity PSTD solve on the GPU (``pstd_elastic_3d``,
    solver/elastic.jl:386-588); same arguments and output as the reference."""
    if kgrid.ndim != 3:
        raise TypeError("MethodError: pstd_elastic_3d takes a KWaveGrid3D")
    return _pstd_elastic(kgrid, medium, source, sensor, pml_size, pml_alpha, progress_callback, context)


class Simulation:
    """A resident simulation: the solve split into create / advance / read (kwb_sim_*)."""

    def __init__(self, kgrid, medium, source, sensor, *, pml_size=20, pml_alpha=2.0,
                 smooth_p0=True, extra_sensors=(), context: Optional[Context] = None):
        self.ctx = context or default_context()
        self.kgrid, self.sensor = kgrid, sensor
        # an ElasticMedium selects the elastic solver (pstd_elastic_2d/3d)
        self.b = build_problem(kgrid, medium, source, sensor, pml_size=pml_size,
                               pml_alpha=pml_alpha, smooth_p0=smooth_p0, extra_sensors=extra_sensors)
        self.Nt = int(self.b.problem.tr.n_cols if self.b.problem.tr.data else self.b.problem.Nt)
        h = C.c_void_p()
        with self.ctx.lock:
            check(self.ctx.lib, self.ctx.handle,
                  self.ctx.lib.kwb_sim_create(self.ctx.handle, C.byref(self.b.problem), C.byref(h)))
        self.handle = h

    def _chk(self, rc):
        return check(self.ctx.lib, self.ctx.handle, rc)

    def advance(self, steps: int):
        self._chk(self.ctx.lib.kwb_sim_advance(self.handle, int(steps)))

    def advance_timed(self, steps: int) -> float:
        ms = C.c_double(0)
        self._chk(self.ctx.lib.kwb_sim_advance_timed(self.handle, int(steps), C.byref(ms)))
        return ms.value

    def sync(self):
        self._chk(self.ctx.lib.kwb_sim_sync(self.handle))

    @property
    def steps_done(self) -> int:
        return int(self.ctx.lib.kwb_sim_steps_done(self.handle))

    def pressure(self) -> np.ndarray:
        n = int(np.prod(self.kgrid.N))
        out = np.empty(n, dtype=np.float32)
        self._chk(self.ctx.lib.kwb_sim_read_pressure(self.handle, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out.reshape(self.kgrid.N, order="F")

    def outputs(self) -> SimulationOutput:
        O, outs, arrays, pfull = _alloc_outputs(self.ctx, self.b, self.kgrid)
        self._chk(self.ctx.lib.kwb_sim_read_outputs(self.handle, C.byref(O)))
        return _collect(self.b, arrays, pfull, self.sensor, self.kgrid, self.Nt)

    def finish(self) -> SimulationOutput:
        """Run the remaining steps and return the outputs (``advance`` to Nt, then ``outputs``),
        with the recorded time series copied back block by block while later steps run
        (kwb_sim_finish)."""
        O, outs, arrays, pfull = _alloc_outputs(self.ctx, self.b, self.kgrid)
        self._chk(self.ctx.lib.kwb_sim_finish(self.handle, C.byref(O)))
        return _collect(self.b, arrays, pfull, self.sensor, self.kgrid, self.Nt)

    def profile(self, steps: int) -> list:
        kt = _lib.KernelTimes()
        self._chk(self.ctx.lib.kwb_sim_profile(self.handle, int(steps), C.byref(kt)))
        return [dict(name=kt.name[i].value.decode(), total_ms=kt.total_ms[i], launches=kt.launches[i],
                     bytes_per_launch=kt.bytes_per_launch[i]) for i in range(kt.n)]

    def info(self):
        nb = C.c_int64(0)
        nl = C.c_int32(0)
        self._chk(self.ctx.lib.kwb_sim_info(self.handle, C.byref(nb), C.byref(nl)))
        return {"device_bytes": nb.value, "launches_per_step": nl.value}

    def schedule(self) -> str:
        """The FFT schedule of this simulation's time step: "tuned" (measured on first use of the
        grid shape), "cache" (an earlier measurement) or "heuristic", then the per-pass choices."""
        buf = C.create_string_buffer(512)
        self._chk(self.ctx.lib.kwb_sim_schedule(self.handle, buf, len(buf)))
        return buf.value.decode()

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.kwb_sim_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------------------
# continuous batching (kwb_submit / kwb_wait): many independent simulations on one GPU
# ---------------------------------------------------------------------------------------------

class Request:
    """A submitted simulation; keeps every host array the C side reads or writes alive."""

    def __init__(self, ctx, ticket, built, O, outs, arrays, pfull, kgrid, sensor, Nt):
        self.ctx, self.ticket = ctx, ticket
        self._keep = (built, O, outs, arrays, pfull)
        self.kgrid, self.sensor, self.Nt = kgrid, sensor, Nt
        self._result = None
        self.info = None

    def done(self) -> bool:
        if self._result is not None or self.info is not None:
            return True
        d = C.c_int32(0)
        check(self.ctx.lib, self.ctx.handle, self.ctx.lib.kwb_poll(self.ctx.handle, self.ticket, C.byref(d)))
        return bool(d.value)

    def result(self, timeout: Optional[float] = None) -> SimulationOutput:
        if self._result is not None:
            return self._result
        if self.info is not None:
            raise KWaveB200Error(self.info["status"], self.info["error"])
        info = _lib.RequestInfo()
        t = -1 if timeout is None else int(timeout * 1e9)
        rc = self.ctx.lib.kwb_wait(self.ctx.handle, self.ticket, t, C.byref(info))
        if rc == _lib.KWB_E_TIMEOUT:
            raise TimeoutError(f"request {self.ticket} still running")
        self.info = dict(status=info.status, submit_ns=info.submit_ns, start_ns=info.start_ns,
                         end_ns=info.end_ns, error=info.error.decode())
        if rc != _lib.KWB_OK:
            raise KWaveB200Error(rc, self.info["error"])
        built, O, outs, arrays, pfull = self._keep
        self._result = _collect(built, arrays, pfull, self.sensor, self.kgrid, self.Nt)
        return self._result

    def cancel(self):
        check(self.ctx.lib, self.ctx.handle, self.ctx.lib.kwb_cancel(self.ctx.handle, self.ticket))

    def __del__(self):
        # The scheduler reads this request's problem arrays and writes its output buffers until it
        # completes: a request dropped unwaited is cancelled and waited for before they are freed.
        try:
            if self._result is None and self.info is None and getattr(self.ctx, "handle", None):
                self.ctx.lib.kwb_cancel(self.ctx.handle, self.ticket)
                self.ctx.lib.kwb_wait(self.ctx.handle, self.ticket, -1, None)
        except Exception:
            pass

    @property
    def latency_s(self) -> Optional[float]:
        return None if self.info is None else (self.info["end_ns"] - self.info["submit_ns"]) / 1e9


class Prepared:
    """A problem packed for the C ABI with its output buffers (host work done ahead of time)."""

    def __init__(self, ctx, kgrid, sensor, built):
        self.ctx, self.kgrid, self.sensor, self.built = ctx, kgrid, sensor, built
        self.Nt = int(built.problem.tr.n_cols if built.problem.tr.data else built.problem.Nt)
        self.O, self.outs, self.arrays, self.pfull = _alloc_outputs(ctx, built, kgrid)

    @property
    def voxels(self) -> int:
        return int(np.prod(self.kgrid.N))


def prepare(kgrid, medium, source, sensor, *, pml_size=20, pml_alpha=2.0, smooth_p0=True,
            extra_sensors=(), context: Optional[Context] = None) -> Prepared:
    ctx = context or default_context()
    b = build_problem(kgrid, medium, source, sensor, pml_size=pml_size, pml_alpha=pml_alpha,
                      smooth_p0=smooth_p0, extra_sensors=extra_sensors)
    return Prepared(ctx, kgrid, sensor, b)


def submit_prepared(prep: Prepared) -> Request:
    ctx = prep.ctx
    t = C.c_uint64(0)
    check(ctx.lib, ctx.handle, ctx.lib.kwb_submit(ctx.handle, C.byref(prep.built.problem), C.byref(prep.O), C.byref(t)))
    return Request(ctx, t.value, prep.built, prep.O, prep.outs, prep.arrays, prep.pfull, prep.kgrid,
                   prep.sensor, prep.Nt)


def solve_prepared(prep: Prepared) -> SimulationOutput:
    """The plain one-at-a-time path: a blocking kwb_solve of a prepared problem."""
    ctx = prep.ctx
    with ctx.lock:
        check(ctx.lib, ctx.handle, ctx.lib.kwb_solve(ctx.handle, C.byref(prep.built.problem), C.byref(prep.O)))
    return _collect(prep.built, prep.arrays, prep.pfull, prep.sensor, prep.kgrid, prep.Nt)


def submit(kgrid, medium, source, sensor, *, pml_size=20, pml_alpha=2.0, smooth_p0=True,
           extra_sensors=(), context: Optional[Context] = None) -> Request:
    """Queue one simulation for continuous batching; returns a Request (non-blocking).  An
    ``ElasticMedium`` queues an elastic solve (the same scheduler serves both solvers)."""
    return submit_prepared(prepare(kgrid, medium, source, sensor, pml_size=pml_size, pml_alpha=pml_alpha,
                                   smooth_p0=smooth_p0, extra_sensors=extra_sensors, context=context))


def serving_config(max_running: int = 64, chunk_steps: int = 32, mem_cap_bytes: int = 0,
                   context: Optional[Context] = None, voxel_budget: Optional[int] = None):
    """Scheduler limits (kwb_serving_config); ``voxel_budget`` (kwb_serving_voxel_budget) caps
    the grid points of the running simulations together (default 4 Mi; 0 = no cap)."""
    ctx = context or default_context()
    check(ctx.lib, ctx.handle, ctx.lib.kwb_serving_config(ctx.handle, max_running, chunk_steps, mem_cap_bytes))
    if voxel_budget is not None:
        check(ctx.lib, ctx.handle, ctx.lib.kwb_serving_voxel_budget(ctx.handle, int(voxel_budget)))


def serving_stats(context: Optional[Context] = None) -> dict:
    ctx = context or default_context()
    st = _lib.ServingStats()
    check(ctx.lib, ctx.handle, ctx.lib.kwb_serving_stats_get(ctx.handle, C.byref(st)))
    return {n: getattr(st, n) for n, _ in st._fields_}


def estimate_device_bytes(kgrid, medium, source, sensor, context: Optional[Context] = None, **kw) -> int:
    ctx = context or default_context()
    b = build_problem(kgrid, medium, source, sensor, **kw)
    v = C.c_int64(0)
    check(ctx.lib, ctx.handle, ctx.lib.kwb_estimate_device_bytes(ctx.handle, C.byref(b.problem), C.byref(v)))
    return v.value


def solve_batch(jobs, context: Optional[Context] = None) -> list:
    """Run many independent simulations together; jobs are (kgrid, medium, source, sensor, kwargs)."""
    reqs = [submit(g, m, s, sen, context=context, **kw) for g, m, s, sen, kw in jobs]
    return [r.result() for r in reqs]


def _job_parts(job):
    """(kgrid, medium, source, sensor, keyword arguments) of one batch entry."""
    if len(job) == 5:
        return job
    kgrid, medium, source, sensor = job
    return kgrid, medium, source, sensor, {}


def run_sharded(jobs, *, world: Optional[int] = None, rank: Optional[int] = None, devices=None,
                runner=None) -> dict:
    """Run a batch of independent simulations over several GPUs; returns {job index: output}
    for the jobs this process ran.

    ``jobs`` is a list of ``(kgrid, medium, source, sensor)`` or ``(..., kwargs)`` entries, the
    arguments of one ``kspace_first_order`` call each.  Jobs are assigned longest first to the
    least-loaded GPU by voxels x steps (``shard_jobs``); simulations are independent, so GPUs
    exchange nothing while they run and the results come together on the host.

    * One process per GPU (torchrun): ``world``/``rank`` (default: torch.distributed's, else 1/0)
      select this process's share, run on device LOCAL_RANK (or ``devices[0]``).
    * One process, several GPUs: ``devices=[0, 1, ...]`` runs every share, one host thread and
      one context per device.

    Each device runs its share through the continuous-batching scheduler (``submit``).
    ``runner(device, built_problems)`` replaces the library call (tests without a GPU)."""
    if world is None or rank is None:
        try:
            import torch.distributed as dist
            ok = dist.is_available() and dist.is_initialized()
        except Exception:
            ok = False
        world = dist.get_world_size() if ok else 1
        rank = dist.get_rank() if ok else 0
    parts = [_job_parts(j) for j in jobs]
    costs = [int(np.prod(g.N)) * int(g.Nt) for g, *_ in parts]

    def run_on(device, idx):
        if runner is not None:
            built = [build_problem(*parts[i][:4], **{k: v for k, v in parts[i][4].items()
                                                     if k in ("pml_size", "pml_alpha", "smooth_p0")})
                     for i in idx]
            return dict(zip(idx, runner(device, built)))
        ctx = Context(device)
        reqs = [submit(*parts[i][:4], context=ctx, **parts[i][4]) for i in idx]
        return {i: r.result() for i, r in zip(idx, reqs)}

    if devices is not None and len(devices) > 1 and world == 1:
        shares = [shard_jobs(costs, len(devices), r) for r in range(len(devices))]
        out, errs = {}, []

        def work(r):
            try:
                out.update(run_on(devices[r], shares[r]))
            except BaseException as e:  # re-raised on the calling thread
                errs.append(e)

        threads = [threading.Thread(target=work, args=(r,)) for r in range(len(devices))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errs:
            raise errs[0]
        return out
    import os
    device = devices[0] if devices else int(os.environ.get("LOCAL_RANK", "0"))
    return run_on(device, shard_jobs(costs, world, rank))


def shard_jobs(costs, world: int, rank: int) -> list:
    """Indices of the jobs rank `rank` runs when `world` GPUs share a batch: longest-processing-
    time-first greedy assignment on the given costs (e.g. voxels x steps).  Simulations are
    independent, so ranks exchange nothing while they run."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]
