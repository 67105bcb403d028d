"""Python surface of the B200 engine.

``LeviathanEngine`` has the constructor and methods of the reference's
pybind11 class ``leviathan_cuda.LeviathanEngine``
(src/bindings/leviathan_pybind11.cpp:82-104) with the same argument meaning:
arrays are converted to the required dtype (the reference binding force-casts,
:32-42), ``step`` releases the GIL while the GPU runs (:44-47, ctypes releases
it for every foreign call), ``get_theta`` returns a new NumPy array (:50-55)
and ``set_theta`` raises ``RuntimeError`` on a size mismatch (:57-65).
Additional methods (``step_n``, ``get_weights``, ``get_state``/``set_state``,
``set_params`` ...) are additive.

``BatchEngine`` runs many independent networks in one launch per step.
"""

from __future__ import annotations

import ctypes as C
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import check

_F32 = np.float32


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data) if a.size else C.c_void_p(0)


def _as(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=dtype)


def variant_info(v: int) -> dict:
    """Tuning parameters of compiled step-kernel variant ``v``."""
    lib = _lib.load()
    u, p, m = C.c_int32(), C.c_int32(), C.c_int32()
    check(lib.lev_variant_info(int(v), C.byref(u), C.byref(p), C.byref(m)))
    return dict(unroll=u.value, pipelined=p.value, min_blocks=m.value)


def pair_variant_info(v: int) -> dict:
    """Tuning parameters of compiled two-steps-per-launch variant ``v``."""
    lib = _lib.load()
    u, m, dp, ln = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
    check(lib.lev_pair_variant_info(int(v), C.byref(u), C.byref(m), C.byref(dp)))
    check(lib.lev_pair_variant_lanes(int(v), C.byref(ln)))
    return dict(unroll=u.value, min_blocks=m.value, deep=dp.value, lanes_per_row=ln.value)


class _EngineBase:
    """Shared handle management and state access of both engine kinds."""

    _h: C.c_void_p

    def __init__(self):
        self._lib = _lib.load()
        self._h = C.c_void_p(0)

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.lev_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        if not self._h.value:
            raise RuntimeError("engine is closed")
        return self._h

    # -- shapes -------------------------------------------------------------
    def _query_shapes(self) -> None:
        n = C.c_int32()
        check(self._lib.lev_num_nets(self.handle, C.byref(n)))
        self.num_nets = n.value
        tn = C.c_int64()
        te = C.c_int64()
        check(self._lib.lev_total_nodes(self.handle, C.byref(tn)))
        check(self._lib.lev_total_edges(self.handle, C.byref(te)))
        self.total_nodes = tn.value
        self.total_edges = te.value
        self.net_N, self.net_E, self.net_max_delay = [], [], []
        for k in range(self.num_nets):
            Nn = C.c_int32()
            En = C.c_int64()
            md = C.c_int32()
            check(self._lib.lev_net_shape(self.handle, k, C.byref(Nn),
                                          C.byref(En), C.byref(md)))
            self.net_N.append(Nn.value)
            self.net_E.append(En.value)
            self.net_max_delay.append(md.value)
        self.node_off = np.concatenate([[0], np.cumsum(self.net_N)]).astype(np.int64)
        self.edge_off = np.concatenate([[0], np.cumsum(self.net_E)]).astype(np.int64)

    # -- stepping -----------------------------------------------------------
    def _step_all(self, dt: float) -> np.ndarray:
        r = np.empty(self.num_nets, dtype=_F32)
        check(self._lib.lev_step(self.handle, C.c_float(dt), _ptr(r)))
        return r

    def _step_n_all(self, dt: float, n: int) -> np.ndarray:
        n = int(n)
        if n < 0:
            raise ValueError("n must be >= 0")
        r = np.empty((n, self.num_nets), dtype=_F32)
        if n:
            check(self._lib.lev_step_n(self.handle, C.c_float(dt), n, _ptr(r)))
        return r

    def step_n_async(self, dt: float, n: int) -> None:
        """Enqueue ``n`` steps and return immediately (r stays on device)."""
        check(self._lib.lev_step_n_async(self.handle, C.c_float(dt), int(n)))

    def synchronize(self) -> None:
        check(self._lib.lev_sync(self.handle))

    @property
    def stream_ptr(self) -> int:
        s = C.c_void_p()
        check(self._lib.lev_get_stream(self.handle, C.byref(s)))
        return s.value or 0

    # -- state --------------------------------------------------------------
    def _get_nodes(self, fn) -> np.ndarray:
        out = np.empty(self.total_nodes, dtype=_F32)
        check(fn(self.handle, _ptr(out)))
        return out

    def get_all_theta(self) -> np.ndarray:
        return self._get_nodes(self._lib.lev_get_theta)

    def set_all_theta(self, theta) -> None:
        t = _as(theta, _F32)
        if t.size != self.total_nodes:
            raise RuntimeError(
                f"theta array size mismatch: expected {self.total_nodes}, got {t.size}")
        check(self._lib.lev_set_theta(self.handle, _ptr(t)))

    def get_weights(self) -> np.ndarray:
        out = np.empty(self.total_edges, dtype=_F32)
        check(self._lib.lev_get_weights(self.handle, _ptr(out)))
        return out

    def reset_weights(self, weights) -> None:
        w = _as(weights, _F32)
        if w.size != self.total_edges:
            raise RuntimeError(
                f"weights array size mismatch: expected {self.total_edges}, got {w.size}")
        check(self._lib.lev_reset_weights(self.handle, _ptr(w)))

    def get_predictor(self):
        th = np.empty(self.total_nodes, dtype=_F32)
        wh = np.empty(self.total_nodes, dtype=_F32)
        check(self._lib.lev_get_predictor(self.handle, _ptr(th), _ptr(wh)))
        return th, wh

    def set_predictor(self, theta_hat=None, omega_hat=None) -> None:
        a = _as(theta_hat, _F32) if theta_hat is not None else None
        b = _as(omega_hat, _F32) if omega_hat is not None else None
        for x in (a, b):
            if x is not None and x.size != self.total_nodes:
                raise RuntimeError("predictor array size mismatch")
        check(self._lib.lev_set_predictor(
            self.handle, _ptr(a) if a is not None else None,
            _ptr(b) if b is not None else None))

    def get_omega(self) -> np.ndarray:
        return self._get_nodes(self._lib.lev_get_omega)

    def set_omega(self, omega) -> None:
        o = _as(omega, _F32)
        if o.size != self.total_nodes:
            raise RuntimeError("omega array size mismatch")
        check(self._lib.lev_set_omega(self.handle, _ptr(o)))

    def get_ring(self, net: int = 0):
        """Delay ring of one network in the reference layout
        ``[N, max_delay+1]`` (leviathan_kernel.cu:142-143) and its slot index
        ``buf_idx`` of the current phase."""
        N = self.net_N[net]
        bs = self.net_max_delay[net] + 1
        out = np.empty((N, bs), dtype=_F32)
        bi = C.c_int32()
        check(self._lib.lev_get_ring(self.handle, int(net), _ptr(out), C.byref(bi)))
        return out, bi.value

    def set_ring(self, ring, buf_idx: int, net: int = 0) -> None:
        N = self.net_N[net]
        bs = self.net_max_delay[net] + 1
        r = _as(ring, _F32)
        if r.shape != (N, bs) and r.size != N * bs:
            raise RuntimeError("ring array size mismatch")
        check(self._lib.lev_set_ring(self.handle, int(net), _ptr(r), int(buf_idx)))

    def step_count(self, net: int = 0) -> int:
        t = C.c_int64()
        check(self._lib.lev_get_step_count(self.handle, int(net), C.byref(t)))
        return t.value

    def get_r(self, net: int = 0) -> float:
        r = C.c_float()
        check(self._lib.lev_get_r(self.handle, int(net), C.byref(r)))
        return r.value

    def _set_gain(self, g: float, net: int) -> None:
        check(self._lib.lev_set_gain(self.handle, int(net), C.c_float(g)))

    def _get_gain(self, net: int) -> float:
        g = C.c_float()
        check(self._lib.lev_get_gain(self.handle, int(net), C.byref(g)))
        return g.value

    def _set_ctrl(self, enabled: bool, net: int) -> None:
        check(self._lib.lev_set_gain_controller(self.handle, int(net), 1 if enabled else 0))

    def set_params(self, net: int = -1, **kw) -> None:
        """Set physics parameters (names of ``LevParams``); unspecified
        fields keep their current value.  ``g`` sets the current gain."""
        cur = self.get_params(0 if net < 0 else net)
        cur.update(kw)
        p = _lib.make_params(**cur)
        check(self._lib.lev_set_params(self.handle, int(net), C.byref(p)))

    def get_params(self, net: int = 0) -> dict:
        p = _lib.LevParams()
        check(self._lib.lev_get_params(self.handle, int(net), C.byref(p)))
        return p.to_dict()

    def set_math_mode(self, mode) -> None:
        if isinstance(mode, str):
            mode = {"reference": 0, "accurate": 1}[mode]
        check(self._lib.lev_set_math_mode(self.handle, int(mode)))

    def get_vram_usage(self) -> int:
        b = C.c_size_t()
        check(self._lib.lev_get_vram_usage(self.handle, C.byref(b)))
        return b.value

    # -- autotuner ----------------------------------------------------------
    def tuning(self) -> list:
        """Degree classes of this engine: tiles, mean slice length, edges and
        the step-kernel variant (unroll, pipelined, min_blocks) in use."""
        out = []
        for c in range(3):
            nt, ml, ed, v = C.c_int32(), C.c_float(), C.c_int64(), C.c_int32()
            check(self._lib.lev_class_info(self.handle, c, C.byref(nt), C.byref(ml),
                                           C.byref(ed), C.byref(v)))
            out.append(dict(cls=c, tiles=nt.value, mean_slice_len=ml.value,
                            edges=ed.value, variant=v.value, **variant_info(v.value)))
        return out

    def autotune(self, dt: float = 0.05, trial_steps: int = 5) -> dict:
        """Time every compiled variant per degree class, keep the fastest;
        the simulation state is restored afterwards."""
        nv = self._lib.lev_num_variants()
        chosen = (C.c_int32 * 3)()
        ms = (C.c_float * (3 * nv))()
        check(self._lib.lev_autotune(self.handle, C.c_float(dt), int(trial_steps),
                                     chosen, ms))
        return dict(chosen=list(chosen),
                    ms=[[ms[c * nv + v] for v in range(nv)] for c in range(3)],
                    variants=[variant_info(v) for v in range(nv)])

    def set_variant(self, cls: int, variant: int) -> None:
        check(self._lib.lev_set_variant(self.handle, int(cls), int(variant)))

    # -- cluster-resident path (small single networks) ---------------------
    def cluster_info(self) -> dict:
        el, en, c, r = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        sm = C.c_int64()
        check(self._lib.lev_cluster_info(self.handle, C.byref(el), C.byref(en), C.byref(c),
                                         C.byref(r), C.byref(sm)))
        return dict(eligible=bool(el.value), enabled=bool(en.value), ctas=c.value,
                    rows_per_cta=r.value, smem_bytes=sm.value)

    def set_cluster_mode(self, enabled: bool) -> None:
        check(self._lib.lev_set_cluster_mode(self.handle, 1 if enabled else 0))

    # -- grid-resident path (mid-sized single networks) --------------------
    def grid_info(self) -> dict:
        el, en, c, r, m = (C.c_int32() for _ in range(5))
        sm = C.c_int64()
        check(self._lib.lev_grid_info(self.handle, C.byref(el), C.byref(en), C.byref(c),
                                      C.byref(r), C.byref(sm), C.byref(m)))
        rows = [R for R in (64, 128, 256) if m.value & R]
        return dict(eligible=bool(el.value), enabled=bool(en.value), ctas=c.value,
                    rows_per_cta=r.value, smem_bytes=sm.value, eligible_rows=rows)

    def set_grid_mode(self, enabled: bool, rows_per_cta: int = 0) -> None:
        """Allow (or forbid) the grid-resident path for step blocks;
        rows_per_cta 64, 128 or 256 picks the CTA size (0 keeps it)."""
        check(self._lib.lev_set_grid_mode(self.handle, 1 if enabled else 0, int(rows_per_cta)))

    def create_profile(self) -> dict:
        """Milliseconds of the phases of this engine's creation (``layout``
        and ``kernel_setup`` run on a helper thread during
        ``staged_uploads``)."""
        ms = (C.c_double * 8)()
        check(self._lib.lev_create_profile(self.handle, ms))
        keys = ("layout", "kernel_setup", "stream_and_device_allocation", "mapped_host_buffer",
                "small_uploads", "staged_uploads", "pack_and_fill_launch", "dma_wait")
        return {k: float(v) for k, v in zip(keys, ms)}

    def set_grid_wait(self, limit_ns: int = 2_000_000_000, extra_arrivals: int = 0) -> None:
        """Bound of the grid-barrier waits (default 2 s).  ``extra_arrivals``
        > 0 makes the next grid-resident block's first wait run out: for
        tests of the timeout path (see ``lev_set_grid_wait``)."""
        check(self._lib.lev_set_grid_wait(self.handle, int(limit_ns), int(extra_arrivals)))

    # -- two steps per launch (step blocks; no zero delays) -----------------
    def pair_info(self) -> list:
        """Per degree class: whether two steps per launch are possible
        (eligible: no zero delay) and in use, the pair variant (-1: one step
        per launch for this class), the autotuner's ms per step of the best
        pair and one-step variants (0 before autotuning)."""
        out = []
        for c in range(3):
            el, en, pv = C.c_int32(), C.c_int32(), C.c_int32()
            pms, sms = C.c_float(), C.c_float()
            check(self._lib.lev_pair_info(self.handle, c, C.byref(el), C.byref(en),
                                          C.byref(pv), C.byref(pms), C.byref(sms)))
            info = dict(cls=c, eligible=bool(el.value), enabled=bool(en.value),
                        pair_variant=pv.value, pair_ms=pms.value, step_ms=sms.value)
            if pv.value >= 0:
                info.update(pair_variant_info(pv.value))
            out.append(info)
        return out

    def set_pair_mode(self, enabled: bool) -> None:
        check(self._lib.lev_set_pair_mode(self.handle, 1 if enabled else 0))

    def set_pair_variant(self, cls: int, variant: int) -> None:
        check(self._lib.lev_set_pair_variant(self.handle, int(cls), int(variant)))

    def time_launches(self, dt: float, n: int = 20) -> tuple:
        """Mean durations (ms) of the two launch phases of a two-step round
        (pair_kernel, finish_kernel -- or two one-step launches), timed with
        CUDA events on the engine stream; advances the simulation 2n steps."""
        ms = (C.c_float * 2)()
        check(self._lib.lev_time_launches(self.handle, C.c_float(dt), int(n), ms))
        return float(ms[0]), float(ms[1])

    # -- checkpoint ---------------------------------------------------------
    def get_state(self) -> dict:
        """Full engine state (the reference exposes no such getter)."""
        th_hat, om_hat = self.get_predictor()
        st = {
            "theta": self.get_all_theta(),
            "theta_hat": th_hat,
            "omega": self.get_omega(),
            "omega_hat": om_hat,
            "weights": self.get_weights(),
            "g": np.array([self._get_gain(k) for k in range(self.num_nets)], _F32),
            "r": np.array([self.get_r(k) for k in range(self.num_nets)], _F32),
            "step": np.array([self.step_count(k) for k in range(self.num_nets)], np.int64),
            "params": [self.get_params(k) for k in range(self.num_nets)],
        }
        rings, bufs = [], []
        for k in range(self.num_nets):
            r, b = self.get_ring(k)
            rings.append(r)
            bufs.append(b)
        st["ring"] = rings
        st["buf_idx"] = np.array(bufs, np.int32)
        return st

    def set_state(self, st: dict) -> None:
        """Restore a state from ``get_state`` (the topology must match)."""
        check(self._lib.lev_set_theta(self.handle, _ptr(_as(st["theta"], _F32))))
        self.set_predictor(st["theta_hat"], st["omega_hat"])
        self.set_omega(st["omega"])
        self.reset_weights(st["weights"])
        for k in range(self.num_nets):
            if "params" in st:
                p = dict(st["params"][k])
                p["g"] = float(st["g"][k])
                self.set_params(k, **p)
            else:
                self._set_gain(float(st["g"][k]), k)
            self.set_ring(st["ring"][k], int(st["buf_idx"][k]), k)


class LeviathanEngine(_EngineBase):
    """Drop-in for ``leviathan_cuda.LeviathanEngine``
    (src/bindings/leviathan_pybind11.cpp:85-104): one network."""

    def __init__(self, N: int, max_delay: int, row_ptr, col_idx, delays,
                 weights, theta, theta_hat, omega, *, params: dict | None = None,
                 math_mode: str | int = "reference"):
        super().__init__()
        N = int(N)
        max_delay = int(max_delay)
        rp = _as(row_ptr, np.int32)
        if rp.size != N + 1:
            raise ValueError(f"row_ptr must have N+1={N + 1} entries, got {rp.size}")
        E = int(rp[-1])
        col = _as(col_idx, np.int32)
        dl = _as(delays, np.uint8)
        w = _as(weights, _F32)
        th = _as(theta, _F32)
        thh = _as(theta_hat, _F32)
        om = _as(omega, _F32)
        for name, arr, n in (("col_idx", col, E), ("delays", dl, E),
                             ("weights", w, E), ("theta", th, N),
                             ("theta_hat", thh, N), ("omega", om, N)):
            if arr.size != n:
                raise ValueError(f"{name} must have {n} entries, got {arr.size}")
        if isinstance(math_mode, str):
            math_mode = {"reference": 0, "accurate": 1}[math_mode]
        p = _lib.make_params(**(params or {}))
        h = C.c_void_p()
        check(self._lib.lev_create(C.byref(h), N, max_delay, _ptr(rp), _ptr(col),
                                   _ptr(dl), _ptr(w), _ptr(th), _ptr(thh), _ptr(om),
                                   C.byref(p), int(math_mode)))
        self._h = h
        self.N = N
        self.max_delay = max_delay
        self.num_edges = E
        self._query_shapes()

    # reference methods (leviathan_pybind11.cpp:90-104)
    def step(self, dt: float) -> float:
        """One step; returns r of the new phases."""
        return float(self._step_all(dt)[0])

    def get_theta(self) -> np.ndarray:
        return self.get_all_theta()

    def set_theta(self, theta) -> None:
        self.set_all_theta(theta)

    def set_gain(self, g: float) -> None:
        self._set_gain(float(g), 0)

    def get_gain(self) -> float:
        return self._get_gain(0)

    def set_gain_controller(self, enabled: bool) -> None:
        self._set_ctrl(bool(enabled), 0)

    # additive
    def step_n(self, dt: float, n: int) -> np.ndarray:
        """``n`` steps in one call (CUDA-graph replay); returns r[n]."""
        return self._step_n_all(dt, n)[:, 0].copy()


class BatchEngine(_EngineBase):
    """Many independent networks (uneven sizes and parameters) advanced
    together, one launch per step over all networks' tiles."""

    def __init__(self, nets: Sequence[dict], *, params: Sequence[dict] | None = None,
                 math_mode: str | int = "reference"):
        super().__init__()
        nets = list(nets)
        if not nets:
            raise ValueError("at least one network is required")
        Ns, mds, rps, cols, dls, ws, ths, thhs, oms = [], [], [], [], [], [], [], [], []
        for k, net in enumerate(nets):
            N = int(net["N"])
            rp = _as(net["row_ptr"], np.int32)
            if rp.size != N + 1:
                raise ValueError(f"network {k}: row_ptr must have N+1 entries")
            E = int(rp[-1])
            arrs = dict(col_idx=_as(net["col_idx"], np.int32),
                        delays=_as(net["delays"], np.uint8),
                        weights=_as(net["weights"], _F32),
                        theta=_as(net["theta"], _F32),
                        theta_hat=_as(net.get("theta_hat", net["theta"]), _F32),
                        omega=_as(net["omega"], _F32))
            for name in ("col_idx", "delays", "weights"):
                if arrs[name].size != E:
                    raise ValueError(f"network {k}: {name} must have {E} entries")
            for name in ("theta", "theta_hat", "omega"):
                if arrs[name].size != N:
                    raise ValueError(f"network {k}: {name} must have {N} entries")
            Ns.append(N)
            mds.append(int(net["max_delay"]))
            rps.append(rp)
            cols.append(arrs["col_idx"])
            dls.append(arrs["delays"])
            ws.append(arrs["weights"])
            ths.append(arrs["theta"])
            thhs.append(arrs["theta_hat"])
            oms.append(arrs["omega"])
        cat = lambda xs, dt: np.ascontiguousarray(np.concatenate(xs), dtype=dt)
        Na = np.array(Ns, np.int32)
        mda = np.array(mds, np.int32)
        rpa = cat(rps, np.int32)
        cola = cat(cols, np.int32)
        dla = cat(dls, np.uint8)
        wa = cat(ws, _F32)
        tha = cat(ths, _F32)
        thha = cat(thhs, _F32)
        oma = cat(oms, _F32)
        if params is None:
            params = [{}] * len(nets)
        if len(params) != len(nets):
            raise ValueError("params must have one entry per network")
        parr = (_lib.LevParams * len(nets))()
        for k, pk in enumerate(params):
            parr[k] = _lib.make_params(**(pk or {}))
        if isinstance(math_mode, str):
            math_mode = {"reference": 0, "accurate": 1}[math_mode]
        h = C.c_void_p()
        check(self._lib.lev_batch_create(
            C.byref(h), len(nets), _ptr(Na), _ptr(mda), _ptr(rpa), _ptr(cola),
            _ptr(dla), _ptr(wa), _ptr(tha), _ptr(thha), _ptr(oma), parr,
            int(math_mode)))
        self._h = h
        self._query_shapes()

    def step(self, dt: float) -> np.ndarray:
        """One step of every network; returns r[num_nets]."""
        return self._step_all(dt)

    def step_n(self, dt: float, n: int) -> np.ndarray:
        """``n`` steps of every network; returns r[n, num_nets]."""
        return self._step_n_all(dt, n)

    def get_theta(self, net: int | None = None) -> np.ndarray:
        if net is None:
            return self.get_all_theta()
        out = np.empty(self.net_N[net], dtype=_F32)
        check(self._lib.lev_get_theta_net(self.handle, int(net), _ptr(out)))
        return out

    def set_theta(self, theta, net: int | None = None) -> None:
        if net is None:
            self.set_all_theta(theta)
            return
        t = _as(theta, _F32)
        if t.size != self.net_N[net]:
            raise RuntimeError("theta array size mismatch")
        check(self._lib.lev_set_theta_net(self.handle, int(net), _ptr(t)))

    def set_gain(self, g, net: int = -1) -> None:
        if np.ndim(g):
            for k, gk in enumerate(g):
                self._set_gain(float(gk), k)
        else:
            self._set_gain(float(g), net)

    def get_gain(self, net: int | None = None):
        if net is None:
            return np.array([self._get_gain(k) for k in range(self.num_nets)], _F32)
        return self._get_gain(net)

    def set_gain_controller(self, enabled: bool, net: int = -1) -> None:
        self._set_ctrl(bool(enabled), net)
