"""Host-side mirror of the reference's channel driver over the C-ABI.

``Channel`` owns one device context (db_init) and exposes the reference's
subroutines by their names: ``fft_xz_to_fourier``, ``fft_xz_to_physical``,
``rk_chan_1``, ``rem_div_chan``, ``apply_bc_vel_post``, ``courant``, plus the
driver's time loop ``step`` (for/diablo.f90:58-69).  Arrays crossing the
boundary use the reference layout (see include/diablo_b200.h).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lib as _L
from .ic import initial_fields, ref_cshape, ref_shape
from .params import DbParams


class Channel:
    def __init__(self, params: DbParams, gy: np.ndarray, stream: int | None = None):
        self.L = _L.load()
        self.p = params.copy()
        self.gy = np.ascontiguousarray(gy, dtype=np.float64)
        if self.gy.shape != (params.ny + 1,):
            raise ValueError(f"gy must hold ny+1 = {params.ny + 1} values")
        h = ctypes.c_void_p()
        rc = self.L.db_init(ctypes.byref(self.p), _L.dptr(self.gy),
                            ctypes.c_void_p(stream) if stream else None, ctypes.byref(h))
        if rc != 0:
            raise _L.DiabloError(rc, self.L.db_last_error(None).decode())
        self.h = h

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.db_finalize(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        _L.check(rc, self.h)

    # -- reference-layout arrays ---------------------------------------------
    def new_real(self) -> np.ndarray:
        return np.zeros(ref_shape(self.p))

    def new_spectral(self) -> np.ndarray:
        return np.zeros(ref_cshape(self.p), dtype=np.complex128)

    @staticmethod
    def _as_d(a: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a)
        return a.view(np.float64) if a.dtype == np.complex128 else a

    def upload_field(self, fid: int, arr: np.ndarray):
        self._ck(self.L.db_upload_field(self.h, fid, _L.dptr(self._as_d(arr).reshape(-1))))

    def download_field(self, fid: int) -> np.ndarray:
        """Spectral fields as reference complex arrays; nu_t / kappa_t
        (LES) as reference real arrays."""
        if fid in (_L.NU_T, _L.KAPPA_T):
            out = self.new_real()
            self._ck(self.L.db_download_field(self.h, fid, _L.dptr(out.reshape(-1))))
            return out
        out = self.new_spectral()
        self._ck(self.L.db_download_field(self.h, fid, _L.dptr(out.view(np.float64).reshape(-1))))
        return out

    def upload_state(self, state: dict):
        for fid in _L.STATE_FIELDS:
            a = state.get(fid)
            if a is None:
                a = self.new_spectral()
            self.upload_field(fid, a)

    def download_state(self) -> dict:
        return {fid: self.download_field(fid) for fid in _L.STATE_FIELDS}

    # -- the reference's subroutines -----------------------------------------
    def fft_xz_to_fourier(self, buf: np.ndarray) -> np.ndarray:
        """In place on a reference-layout real array; returns its complex view."""
        assert buf.dtype == np.float64 and buf.flags["C_CONTIGUOUS"]
        self._ck(self.L.db_fft_xz_to_fourier(self.h, _L.dptr(buf.reshape(-1))))
        return buf.reshape(-1).view(np.complex128).reshape(ref_cshape(self.p))

    def fft_xz_to_physical(self, cbuf: np.ndarray) -> np.ndarray:
        """In place on a reference-layout complex array; returns its real view."""
        d = cbuf.view(np.float64) if cbuf.dtype == np.complex128 else cbuf
        assert d.flags["C_CONTIGUOUS"]
        self._ck(self.L.db_fft_xz_to_physical(self.h, _L.dptr(d.reshape(-1))))
        return d.reshape(-1).reshape(ref_shape(self.p))

    def fft_xz_to_fourier_dev(self, t) -> None:
        """In place on a device reference-layout real array (a contiguous
        float64 CUDA tensor), ordered on the context's stream."""
        assert t.is_cuda and t.dtype.is_floating_point and t.element_size() == 8 and t.is_contiguous()
        self._ck(self.L.db_fft_xz_to_fourier_dev(self.h, ctypes.c_void_p(t.data_ptr())))

    def fft_xz_to_physical_dev(self, t) -> None:
        """In place on a device reference-layout complex array (a contiguous
        complex128 or float64 CUDA tensor), ordered on the context's stream."""
        assert t.is_cuda and t.element_size() in (8, 16) and t.is_contiguous()
        self._ck(self.L.db_fft_xz_to_physical_dev(self.h, ctypes.c_void_p(t.data_ptr())))

    def rk_chan_1(self, rk_step: int):
        self._ck(self.L.db_rk_substep(self.h, rk_step))

    def step(self, nsteps: int = 1):
        """nsteps driver steps: time_step += 1, three substeps, time += dt."""
        self._ck(self.L.db_rk_steps(self.h, nsteps))

    def rem_div_chan(self):
        self._ck(self.L.db_rem_div(self.h))

    def poisson_p_chan(self):
        """cp from the velocity and buoyancy (restart without pressure)."""
        self._ck(self.L.db_poisson_p(self.h))

    def apply_bc_vel_post(self):
        self._ck(self.L.db_apply_bc_vel_post(self.h))

    def courant(self) -> float:
        dt = ctypes.c_double()
        self._ck(self.L.db_courant(self.h, ctypes.byref(dt)))
        return dt.value

    def divergence(self) -> float:
        d = ctypes.c_double()
        self._ck(self.L.db_divergence(self.h, ctypes.byref(d)))
        return d.value

    def stats(self) -> dict:
        """Mean and energy-budget profiles (save_stats_chan), FP64: a dict of
        arrays over the planes 0..Nyp+1 (see include/diablo_b200.h, db_stats)."""
        out = np.zeros((len(_L.STAT_ROWS), self.p.ny + 2))
        self._ck(self.L.db_stats(self.h, _L.dptr(out.reshape(-1))))
        return {k: out[i].copy() for i, k in enumerate(_L.STAT_ROWS)}

    def budget(self) -> dict:
        """Energy-budget rows that need the mean flow as a function of x
        (compute_TKE, compute_TKE_Production, compute_MKE_diss,
        compute_Vorticity), FP64: a dict of arrays over the planes 0..Nyp+1
        (see include/diablo_b200.h, db_budget)."""
        out = np.zeros((len(_L.BUDGET_ROWS), self.p.ny + 2))
        self._ck(self.L.db_budget(self.h, _L.dptr(out.reshape(-1))))
        return {k: out[i].copy() for i, k in enumerate(_L.BUDGET_ROWS)}

    def bpe(self, nbin: int | None = None):
        """(BPE, PDF[nbin], bin edges[nbin + 1]) of compute_BPE; nbin
        defaults to Nx as in the reference."""
        n = int(nbin or self.p.nx)
        pdf, edges, e = np.zeros(n), np.zeros(n + 1), ctypes.c_double()
        self._ck(self.L.db_bpe(self.h, n, _L.dptr(pdf), _L.dptr(edges), ctypes.byref(e)))
        return e.value, pdf, edges

    def bin_ystar(self, field=None, nbin: int | None = None):
        """Bin_Ystar_and_Write: (binned field, bin weights) over the
        buoyancy bins of compute_BPE.  field: a physical array in the
        reference layout (Nyp+2, Nz+2, Nx+2); None bins the kinetic energy
        0.5 (u1^2 + u2^2 + u3^2) of the current state (KE_zstar)."""
        n = int(nbin or self.p.nx)
        out, w = np.zeros(n), np.zeros(n)
        if field is None:
            self._ck(self.L.db_bin_ystar(self.h, _L.DB_ZS_KE, None, n, _L.dptr(out), _L.dptr(w)))
        else:
            f = np.ascontiguousarray(field, np.float64)
            assert f.shape == (self.p.ny + 2, self.p.nz + 2, self.p.nx + 2), f.shape
            self._ck(self.L.db_bin_ystar(self.h, _L.DB_ZS_FIELD, _L.dptr(f.reshape(-1)), n, _L.dptr(out),
                                         _L.dptr(w)))
        return out, w

    def les_stats(self) -> dict:
        """The LES statistics (save_stats_LES_OOL's nu_sgs, kappa_sgs and
        compute_TKE_diss_les's eps_sgs2), FP64: a dict of arrays over the
        planes 0..Nyp+1 from the stored nu_t, kappa_t (les_eval() first
        for those of the current state)."""
        out = np.zeros((len(_L.LES_ROWS), self.p.ny + 2))
        self._ck(self.L.db_les_stats(self.h, _L.dptr(out.reshape(-1))))
        return {k: out[i].copy() for i, k in enumerate(_L.LES_ROWS)}

    def set_sgs_net(self, net):
        """Learned closure for les_model_type 6 (a SgsNet that outlives this channel)."""
        self._sgs = net
        self._ck(self.L.db_set_sgs_net(self.h, net.h if net is not None else None))

    def les_eval(self, model: int = 5, features: bool = False):
        """The SGS model on the current state: (nu_t, kappa_t) in the
        reference physical layout, and the closure features
        [Nyp+2][Nz][Nx][16] when asked."""
        nu, ka = self.new_real(), self.new_real()
        f = np.zeros((self.p.ny + 2, self.p.nz, self.p.nx, 16), np.float32) if features else None
        self._ck(self.L.db_les_eval(self.h, model, _L.dptr(nu.reshape(-1)), _L.dptr(ka.reshape(-1)),
                                    _L.fptr(f.reshape(-1)) if f is not None else None))
        return (nu, ka, f) if features else (nu, ka)

    def sgs_targets(self, gy_coarse, fx: int = 4, fy: int = 4, fz: int = 4):
        """Box-filtered training data of the learned closure from this
        (resolved) state: CUDA tensors (features [n][16], targets [n][2])."""
        import torch
        g = np.ascontiguousarray(gy_coarse, np.float64)
        n = ctypes.c_longlong()
        self._ck(self.L.db_sgs_targets(self.h, fx, fy, fz, _L.dptr(g), None, None, ctypes.byref(n)))
        feat = torch.empty((n.value, 16), dtype=torch.float32, device="cuda")
        tgt = torch.empty((n.value, 2), dtype=torch.float32, device="cuda")
        self._ck(self.L.db_sgs_targets(self.h, fx, fy, fz, _L.dptr(g), ctypes.c_void_p(feat.data_ptr()),
                                       ctypes.c_void_p(tgt.data_ptr()), ctypes.byref(n)))
        return feat, tgt

    def autotune(self) -> str:
        """Pick launch shapes by timing them on this context; returns the report."""
        buf = ctypes.create_string_buffer(4096)
        self._ck(self.L.db_autotune(self.h, buf, len(buf)))
        return buf.value.decode()

    def tuning(self) -> list:
        """The launch shapes in use (db_get_tuning order)."""
        v = (ctypes.c_int * _L.NTUNE)()
        self._ck(self.L.db_get_tuning(self.h, v, _L.NTUNE))
        return list(v)

    def set_tuning(self, shapes) -> None:
        """Set launch shapes (db_get_tuning order; 0 = built-in default)."""
        v = (ctypes.c_int * _L.NTUNE)(*[int(x) for x in shapes])
        self._ck(self.L.db_set_tuning(self.h, v, _L.NTUNE))

    def set_clock(self, time=0.0, time_step=0, save_stats_time=1e300, save_flow_time=1e300):
        self._ck(self.L.db_set_clock(self.h, time, time_step, save_stats_time, save_flow_time))

    def clear_status(self) -> None:
        """Clear the accumulated DB_FLAG_* bits."""
        self._ck(self.L.db_clear_status(self.h))

    def set_wait_limit(self, polls: int) -> None:
        """Failure-handling hook for tests: polls of the first wait on each
        TMA copy before it gives up (0 = built-in bound); db_set_wait_limit."""
        self._ck(self.L.db_set_wait_limit(self.h, int(polls)))

    def status(self) -> _L.DbStatus:
        s = _L.DbStatus()
        self._ck(self.L.db_get_status(self.h, ctypes.byref(s)))
        return s

    # -- create_flow_chan ------------------------------------------------------
    def init_flow(self, seed: int = 0, noise: str = "gaussian", fields=None):
        """Initial condition as create_flow_chan/create_th_chan build it
        (for/flow.f90:260-499, 562-659): physical fields -> Fourier,
        apply_BC_vel_mpi_post, rem_div_chan; cp from a zero pressure."""
        u1, u2, u3, th = fields if fields is not None else initial_fields(self.p, self.gy, seed, noise)
        spec = {}
        for fid, a in ((_L.CU1, u1), (_L.CU2, u2), (_L.CU3, u3), (_L.CTH, th)):
            b = np.ascontiguousarray(a, dtype=np.float64).copy()
            spec[fid] = self.fft_xz_to_fourier(b).copy()
        self.upload_state(spec)
        self.apply_bc_vel_post()
        self.rem_div_chan()
