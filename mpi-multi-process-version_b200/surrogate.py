"""The warm-start surrogate network on the GPU: a 4-level U-Net (~1.95 M
parameters; bf16 weights and activations, FP32 accumulation, gradients and
Adam state) whose every pass runs on this library's own kernels
(include/lbm_surrogate.h).  torch provides device memory and the stream only.

The reference has no learned component: it always starts from the conduction
state of initial() (natural-convection_2dim_mono.f90:199-240).  The network
maps (Ra, Pr, grid-coordinate maps) to a steady (u, v, T) field that
lbm_init_warm turns into populations.

Layers (3x3 convolutions with SiLU; "|" is a channel concatenation held in one
buffer, the upsampled part first):

    e1a 32->32, e1b 32->32 = s1        R x R
    pool; e2a 32->64, e2b 64->64 = s2  R/2
    pool; e3a 64->128, e3b = s3        R/4
    pool; ba 128->256, bb 256->256     R/8
    up | s3: d3a 384->128, d3b         R/4
    up | s2: d2a 192->64, d2b          R/2
    up | s1: d1a 96->32, d1b           R
    head 1x1 32->3 (linear)
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lbm as L

IN_CH = 32
LEVELS = (32, 64, 128, 256)
OUT_CH = 3

_dp = ctypes.c_void_p
_i64, _i32, _f32 = ctypes.c_int64, ctypes.c_int32, ctypes.c_float

_SIGS = {
    "lbm_nn_conv3x3": [_dp, _i64, _i32, _dp, _dp, _i32, _i32, _i32, _i32, _i32, _dp, _i64, _i32, _i32, _dp, _i64,
                       _i32, _i32, _dp],
    "lbm_nn_flip_weights": [_dp, _dp, _i32, _i32, _dp],
    "lbm_nn_wgrad_workspace": [_i32, _i32, _i32, _i32, _i32],
    "lbm_nn_conv3x3_wgrad": [_dp, _dp, _i64, _i32, _i32, _i32, _i32, _i32, _i32, _dp, _i64, _dp, _dp],
    "lbm_nn_colsum_workspace": [_i64, _i32],
    "lbm_nn_colsum": [_dp, _i64, _i32, _dp, _dp, _dp],
    "lbm_nn_silu_backward": [_dp, _i64, _i32, _dp, _i64, _i32, _dp, _dp],
    "lbm_nn_pool2": [_dp, _i64, _i32, _i32, _i32, _i32, _i32, _dp, _i64, _i32, _dp],
    "lbm_nn_pool2_backward": [_dp, _i64, _i32, _i32, _i32, _i32, _i32, _dp, _i64, _i32, _dp],
    "lbm_nn_up2": [_dp, _i64, _i32, _i32, _i32, _i32, _i32, _dp, _i64, _i32, _dp],
    "lbm_nn_up2_backward": [_dp, _i64, _i32, _i32, _i32, _i32, _i32, _dp, _i64, _i32, _i32, _dp],
    "lbm_nn_head": [_dp, _i64, _i32, _dp, _dp, _i64, _i32, _i32, _dp, _dp],
    "lbm_nn_head_workspace": [_i64, _i32, _i32],
    "lbm_nn_head_backward": [_dp, _dp, _i64, _i32, _dp, _i64, _i32, _i32, _dp, _i64, _i32, _dp, _i64, _dp, _dp, _dp],
    "lbm_nn_mse_workspace": [_i64, _i32],
    "lbm_nn_mse": [_dp, _dp, _dp, _i64, _i32, _dp, _dp, _i64, _dp, _dp],
    "lbm_nn_adam": [_dp, _dp, _dp, _dp, _dp, _i64, _f32, _f32, _f32, _f32, _f32, _f32, _f32, _dp],
    "lbm_nn_to_bf16": [_dp, _dp, _i64, _dp],
    "lbm_nn_set_tensor_path": [_i32],
    "lbm_nn_get_tensor_path": [],
    "lbm_nn_timeouts": [_dp, _i32],
}
NN_EXPORTS = list(_SIGS)


def set_tensor_path(path):
    """0: mma.sync convolutions (the default); 1: tcgen05 (TMEM accumulators)."""
    _chk(nn().lbm_nn_set_tensor_path(int(path)), "lbm_nn_set_tensor_path")


def tensor_path():
    return int(nn().lbm_nn_get_tensor_path())


def timeouts(reset=False):
    c = ctypes.c_int32()
    _chk(nn().lbm_nn_timeouts(ctypes.byref(c), int(bool(reset))), "lbm_nn_timeouts")
    return int(c.value)

_bound = False


def nn():
    """The library with the surrogate entry points typed."""
    global _bound
    lib = L.lib()
    if not _bound:
        for name, args in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int64 if name.endswith("_workspace") else ctypes.c_int
        _bound = True
    return lib


def _chk(st, what):
    if st != 0:
        raise L.LBMError(st, f"{what}: {L.lib().lbm_last_error().decode()}")


def layer_table():
    """[(name, Cin, Cout)] of the 3x3 layers in execution order."""
    c1, c2, c3, c4 = LEVELS
    return [("e1a", IN_CH, c1), ("e1b", c1, c1), ("e2a", c1, c2), ("e2b", c2, c2),
            ("e3a", c2, c3), ("e3b", c3, c3), ("ba", c3, c4), ("bb", c4, c4),
            ("d3a", c4 + c3, c3), ("d3b", c3, c3), ("d2a", c3 + c2, c2), ("d2b", c2, c2),
            ("d1a", c2 + c1, c1), ("d1b", c1, c1)]


def _align(n, a=64):
    return (n + a - 1) // a * a


class Net:
    """Parameters (flat FP32 master, bf16 copy, gradients, Adam moments) and
    per-batch-size activation buffers of the U-Net, on one CUDA device."""

    def __init__(self, R=128, device=0, seed=0, params=None):
        import torch
        self.torch = torch
        if R % 8 or R < 16:
            raise ValueError("R must be a multiple of 8, >= 16")
        self.R = R
        self.dev = torch.device("cuda", device)
        self.table = layer_table()
        off, self.off = 0, {}
        for name, ci, co in self.table:
            self.off[name] = (off, _align(off + 9 * ci * co))
            off = _align(self.off[name][1] + co)
        self.off["head"] = (off, _align(off + OUT_CH * LEVELS[0]))
        self.n_params_padded = _align(self.off["head"][1] + OUT_CH)
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.master = torch.zeros(self.n_params_padded, **f32)
        self.grad = torch.zeros_like(self.master)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.pb = torch.zeros(self.n_params_padded, dtype=torch.bfloat16, device=self.dev)
        self.wt = torch.zeros_like(self.pb)
        self.t = 0
        self.set_params(params if params is not None else init_params(seed))
        self._bufs = {}
        self.stream = torch.cuda.current_stream(self.dev)
        self.launches = 0

    # -- parameters -------------------------------------------------------
    @property
    def n_params(self):
        return sum(9 * ci * co + co for _, ci, co in self.table) + OUT_CH * LEVELS[0] + OUT_CH

    def set_params(self, params):
        """params: {name: (w (Cout, 9, Cin), b (Cout,))} plus 'head': (wh (3, 32), bh (3,))."""
        host = np.zeros(self.n_params_padded, dtype=np.float32)
        for name, ci, co in self.table:
            w, b = params[name]
            o, ob = self.off[name]
            host[o:o + 9 * ci * co] = np.asarray(w, dtype=np.float32).reshape(-1)
            host[ob:ob + co] = np.asarray(b, dtype=np.float32)
        wh, bh = params["head"]
        o, ob = self.off["head"]
        host[o:o + wh.size] = np.asarray(wh, dtype=np.float32).reshape(-1)
        host[ob:ob + OUT_CH] = np.asarray(bh, dtype=np.float32)
        self.master.copy_(self.torch.from_numpy(host))
        _chk(nn().lbm_nn_to_bf16(self.master.data_ptr(), self.pb.data_ptr(), self.n_params_padded, self._s()),
             "lbm_nn_to_bf16")

    def get_params(self, which="master"):
        src = {"master": self.master, "grad": self.grad}[which]
        host = src.detach().cpu().numpy()
        out = {}
        for name, ci, co in self.table:
            o, ob = self.off[name]
            out[name] = (host[o:o + 9 * ci * co].reshape(co, 9, ci).copy(), host[ob:ob + co].copy())
        o, ob = self.off["head"]
        out["head"] = (host[o:o + OUT_CH * LEVELS[0]].reshape(OUT_CH, LEVELS[0]).copy(), host[ob:ob + OUT_CH].copy())
        return out

    def state_dict(self):
        return {"R": self.R, "t": self.t, "master": self.master.cpu().numpy(), "m": self.m.cpu().numpy(),
                "v": self.v.cpu().numpy()}

    def load_state(self, master, m=None, v=None, t=0):
        self.master.copy_(self.torch.from_numpy(np.asarray(master, dtype=np.float32)))
        if m is not None:
            self.m.copy_(self.torch.from_numpy(np.asarray(m, dtype=np.float32)))
            self.v.copy_(self.torch.from_numpy(np.asarray(v, dtype=np.float32)))
        self.t = int(t)
        _chk(nn().lbm_nn_to_bf16(self.master.data_ptr(), self.pb.data_ptr(), self.n_params_padded, self._s()),
             "lbm_nn_to_bf16")

    # -- pointers ---------------------------------------------------------
    def _s(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def _w(self, name, flipped=False):
        t = self.wt if flipped else self.pb
        return t.data_ptr() + 2 * self.off[name][0]

    def _b(self, name):
        return self.master.data_ptr() + 4 * self.off[name][1]

    def _gw(self, name):
        return self.grad.data_ptr() + 4 * self.off[name][0]

    def _gb(self, name):
        return self.grad.data_ptr() + 4 * self.off[name][1]

    # -- buffers ----------------------------------------------------------
    def buffers(self, B):
        """Activation and gradient buffers for batch size B (allocated once)."""
        if B in self._bufs:
            return self._bufs[B]
        torch = self.torch
        R = self.R
        c1, c2, c3, c4 = LEVELS
        bf = dict(dtype=torch.bfloat16, device=self.dev)
        f32 = dict(dtype=torch.float32, device=self.dev)
        res = {"e1a": R, "e1b": R, "e2a": R // 2, "e2b": R // 2, "e3a": R // 4, "e3b": R // 4, "ba": R // 8,
               "bb": R // 8, "d3a": R // 4, "d3b": R // 4, "d2a": R // 2, "d2b": R // 2, "d1a": R, "d1b": R}
        b = {"res": res}
        b["x"] = torch.zeros(B, R, R, IN_CH, **bf)
        b["cat1"] = torch.zeros(B, R, R, c2 + c1, **bf)
        b["cat2"] = torch.zeros(B, R // 2, R // 2, c3 + c2, **bf)
        b["cat3"] = torch.zeros(B, R // 4, R // 4, c4 + c3, **bf)
        b["p1"] = torch.zeros(B, R // 2, R // 2, c1, **bf)
        b["p2"] = torch.zeros(B, R // 4, R // 4, c2, **bf)
        b["p3"] = torch.zeros(B, R // 8, R // 8, c3, **bf)
        for name, ci, co in self.table:
            r = res[name]
            b["z_" + name] = torch.zeros(B, r, r, co, **f32)
            b["a_" + name] = torch.zeros(B, r, r, co, **bf)   # unused for layers writing into a concat buffer
            b["da_" + name] = torch.zeros(B, r, r, co, **f32)
            b["dz_" + name] = torch.zeros(B, r, r, co, **bf)
        b["y"] = torch.zeros(B * R * R, OUT_CH, **f32)
        b["dy"] = torch.zeros(B * R * R, OUT_CH, **f32)
        b["dcat1"] = torch.zeros(B, R, R, c2 + c1, **f32)
        b["dcat2"] = torch.zeros(B, R // 2, R // 2, c3 + c2, **f32)
        b["dcat3"] = torch.zeros(B, R // 4, R // 4, c4 + c3, **f32)
        b["dp1"] = torch.zeros(B, R // 2, R // 2, c1, **f32)
        b["dp2"] = torch.zeros(B, R // 4, R // 4, c2, **f32)
        b["dp3"] = torch.zeros(B, R // 8, R // 8, c3, **f32)
        lib = nn()
        ws = max(lib.lbm_nn_wgrad_workspace(B, res[n], res[n], ci, co) for n, ci, co in self.table)
        ws = max(ws, max(lib.lbm_nn_colsum_workspace(B * res[n] * res[n], co) for n, ci, co in self.table))
        ws = max(ws, lib.lbm_nn_head_workspace(B * R * R, c1, OUT_CH), lib.lbm_nn_mse_workspace(B * R * R, OUT_CH))
        b["ws"] = torch.zeros(int(ws), **f32)
        b["loss"] = torch.zeros(1, **f32)
        self._bufs[B] = b
        return b

    # -- kernels ----------------------------------------------------------
    def _conv(self, B, name, x, xs, xo, of, os_, oo, acc, oa, as_, ao, act, bias, flipped, H, Cin, Cout):
        st = nn().lbm_nn_conv3x3(x, xs, xo, self._w(name, flipped), self._b(name) if bias else None, B, H, H, Cin,
                                 Cout, of, os_, oo, acc, oa, as_, ao, act, self._s())
        _chk(st, f"conv {name}")

    def forward(self, x=None, B=None):
        """Forward pass on buffers(B)['x'] (or copy x, a bf16 (B, R, R, 32)
        tensor, there first).  Returns the FP32 output (B*R*R, 3)."""
        if x is not None:
            B = x.shape[0]
            self.buffers(B)["x"].copy_(x)
        b = self.buffers(B)
        R = self.R
        c1, c2, c3, c4 = LEVELS
        lib = nn()
        s = self._s()
        # (name, input ptr, stride, offset, output bf16 ptr, stride, offset)
        plan = [
            ("e1a", b["x"], IN_CH, 0, b["a_e1a"], c1, 0),
            ("e1b", b["a_e1a"], c1, 0, b["cat1"], c2 + c1, c2),
            ("e2a", b["p1"], c1, 0, b["a_e2a"], c2, 0),
            ("e2b", b["a_e2a"], c2, 0, b["cat2"], c3 + c2, c3),
            ("e3a", b["p2"], c2, 0, b["a_e3a"], c3, 0),
            ("e3b", b["a_e3a"], c3, 0, b["cat3"], c4 + c3, c4),
            ("ba", b["p3"], c3, 0, b["a_ba"], c4, 0),
            ("bb", b["a_ba"], c4, 0, b["a_bb"], c4, 0),
            ("d3a", b["cat3"], c4 + c3, 0, b["a_d3a"], c3, 0),
            ("d3b", b["a_d3a"], c3, 0, b["a_d3b"], c3, 0),
            ("d2a", b["cat2"], c3 + c2, 0, b["a_d2a"], c2, 0),
            ("d2b", b["a_d2a"], c2, 0, b["a_d2b"], c2, 0),
            ("d1a", b["cat1"], c2 + c1, 0, b["a_d1a"], c1, 0),
            ("d1b", b["a_d1a"], c1, 0, b["a_d1b"], c1, 0),
        ]
        tab = {n: (ci, co) for n, ci, co in self.table}
        for name, xin, xs, xo, oa, as_, ao in plan:
            ci, co = tab[name]
            H = b["res"][name]
            self._conv(B, name, xin.data_ptr(), xs, xo, b["z_" + name].data_ptr(), co, 0, 0, oa.data_ptr(), as_, ao,
                       1, True, False, H, ci, co)
            if name == "e1b":
                _chk(lib.lbm_nn_pool2(b["cat1"].data_ptr(), c2 + c1, c2, B, R, R, c1, b["p1"].data_ptr(), c1, 0, s), "pool")
            elif name == "e2b":
                _chk(lib.lbm_nn_pool2(b["cat2"].data_ptr(), c3 + c2, c3, B, R // 2, R // 2, c2, b["p2"].data_ptr(), c2, 0,
                                      s), "pool")
            elif name == "e3b":
                _chk(lib.lbm_nn_pool2(b["cat3"].data_ptr(), c4 + c3, c4, B, R // 4, R // 4, c3, b["p3"].data_ptr(), c3, 0,
                                      s), "pool")
            elif name == "bb":
                _chk(lib.lbm_nn_up2(b["a_bb"].data_ptr(), c4, 0, B, R // 8, R // 8, c4, b["cat3"].data_ptr(), c4 + c3, 0,
                                    s), "up")
            elif name == "d3b":
                _chk(lib.lbm_nn_up2(b["a_d3b"].data_ptr(), c3, 0, B, R // 4, R // 4, c3, b["cat2"].data_ptr(), c3 + c2, 0,
                                    s), "up")
            elif name == "d2b":
                _chk(lib.lbm_nn_up2(b["a_d2b"].data_ptr(), c2, 0, B, R // 2, R // 2, c2, b["cat1"].data_ptr(), c2 + c1, 0,
                                    s), "up")
        o, ob = self.off["head"]
        _chk(lib.lbm_nn_head(b["a_d1b"].data_ptr(), c1, 0, self.pb.data_ptr() + 2 * o, self.master.data_ptr() + 4 * ob,
                             B * R * R, c1, OUT_CH, b["y"].data_ptr(), s), "head")
        self.launches += 14 + 7
        return b["y"]

    def loss(self, target, B, weights=None):
        """MSE of buffers(B)['y'] against target (FP32 (B*R*R, 3)); writes dy."""
        b = self.buffers(B)
        P = B * self.R * self.R
        _chk(nn().lbm_nn_mse(b["y"].data_ptr(), target.data_ptr(), weights.data_ptr() if weights is not None else None,
                             P, OUT_CH, b["dy"].data_ptr(), b["ws"].data_ptr(), b["ws"].numel(), b["loss"].data_ptr(),
                             self._s()), "mse")
        self.launches += 2
        return b["loss"]

    def backward(self, B):
        """Gradients of sum(dy * y) (dy in buffers(B)['dy']) into self.grad."""
        b = self.buffers(B)
        R = self.R
        c1, c2, c3, c4 = LEVELS
        lib = nn()
        s = self._s()
        tab = {n: (ci, co) for n, ci, co in self.table}
        for name, ci, co in self.table:
            _chk(lib.lbm_nn_flip_weights(self._w(name), self._w(name, True), co, ci, s), "flip")
        ws, wsn = b["ws"].data_ptr(), b["ws"].numel()
        o, ob = self.off["head"]
        _chk(lib.lbm_nn_head_backward(b["dy"].data_ptr(), b["a_d1b"].data_ptr(), c1, 0, self.pb.data_ptr() + 2 * o,
                                      B * R * R, c1, OUT_CH, b["da_d1b"].data_ptr(), c1, 0, ws, wsn,
                                      self.grad.data_ptr() + 4 * o, self.grad.data_ptr() + 4 * ob, s), "head backward")

        def back(name, da_ptr, das, dao, x_ptr, xs, xo, dx_ptr=None, dxs=0, dxo=0, dx_acc=0):
            ci, co = tab[name]
            H = b["res"][name]
            P = B * H * H
            dz = b["dz_" + name]
            _chk(lib.lbm_nn_silu_backward(da_ptr, das, dao, b["z_" + name].data_ptr(), P, co, dz.data_ptr(), s),
                 "silu backward")
            _chk(lib.lbm_nn_conv3x3_wgrad(dz.data_ptr(), x_ptr, xs, xo, B, H, H, ci, co, ws, wsn, self._gw(name), s),
                 f"wgrad {name}")
            _chk(lib.lbm_nn_colsum(dz.data_ptr(), P, co, ws, self._gb(name), s), f"bias grad {name}")
            if dx_ptr is not None:
                self._conv(B, name, dz.data_ptr(), co, 0, dx_ptr, dxs, dxo, dx_acc, None, 0, 0, 0, False, True, H, co, ci)

        p = lambda key: b[key].data_ptr()  # noqa: E731
        back("d1b", p("da_d1b"), c1, 0, p("a_d1a"), c1, 0, p("da_d1a"), c1, 0)
        back("d1a", p("da_d1a"), c1, 0, p("cat1"), c2 + c1, 0, p("dcat1"), c2 + c1, 0)
        _chk(lib.lbm_nn_up2_backward(p("dcat1"), c2 + c1, 0, B, R // 2, R // 2, c2, p("da_d2b"), c2, 0, 0, s), "up bwd")
        back("d2b", p("da_d2b"), c2, 0, p("a_d2a"), c2, 0, p("da_d2a"), c2, 0)
        back("d2a", p("da_d2a"), c2, 0, p("cat2"), c3 + c2, 0, p("dcat2"), c3 + c2, 0)
        _chk(lib.lbm_nn_up2_backward(p("dcat2"), c3 + c2, 0, B, R // 4, R // 4, c3, p("da_d3b"), c3, 0, 0, s), "up bwd")
        back("d3b", p("da_d3b"), c3, 0, p("a_d3a"), c3, 0, p("da_d3a"), c3, 0)
        back("d3a", p("da_d3a"), c3, 0, p("cat3"), c4 + c3, 0, p("dcat3"), c4 + c3, 0)
        _chk(lib.lbm_nn_up2_backward(p("dcat3"), c4 + c3, 0, B, R // 8, R // 8, c4, p("da_bb"), c4, 0, 0, s), "up bwd")
        back("bb", p("da_bb"), c4, 0, p("a_ba"), c4, 0, p("da_ba"), c4, 0)
        back("ba", p("da_ba"), c4, 0, p("p3"), c3, 0, p("dp3"), c3, 0)
        _chk(lib.lbm_nn_pool2_backward(p("dp3"), c3, 0, B, R // 4, R // 4, c3, p("dcat3"), c4 + c3, c4, s), "pool bwd")
        back("e3b", p("dcat3"), c4 + c3, c4, p("a_e3a"), c3, 0, p("da_e3a"), c3, 0)
        back("e3a", p("da_e3a"), c3, 0, p("p2"), c2, 0, p("dp2"), c2, 0)
        _chk(lib.lbm_nn_pool2_backward(p("dp2"), c2, 0, B, R // 2, R // 2, c2, p("dcat2"), c3 + c2, c3, s), "pool bwd")
        back("e2b", p("dcat2"), c3 + c2, c3, p("a_e2a"), c2, 0, p("da_e2a"), c2, 0)
        back("e2a", p("da_e2a"), c2, 0, p("p1"), c1, 0, p("dp1"), c1, 0)
        _chk(lib.lbm_nn_pool2_backward(p("dp1"), c1, 0, B, R, R, c1, p("dcat1"), c2 + c1, c2, s), "pool bwd")
        back("e1b", p("dcat1"), c2 + c1, c2, p("a_e1a"), c1, 0, p("da_e1a"), c1, 0)
        back("e1a", p("da_e1a"), c1, 0, p("x"), IN_CH, 0)
        self.launches += 14 + 3 + 13 * 6 + 5 + 3 + 3

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        self.t += 1
        c1, c2 = 1.0 - b1 ** self.t, 1.0 - b2 ** self.t
        _chk(nn().lbm_nn_adam(self.master.data_ptr(), self.pb.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
                              self.v.data_ptr(), self.n_params_padded, lr, b1, b2, eps, c1, c2, wd, self._s()), "adam")
        self.launches += 1


def init_params(seed=0):
    """He-normal weights, zero biases (numpy, seeded)."""
    rng = np.random.default_rng(seed)
    params = {}
    for name, ci, co in layer_table():
        params[name] = (rng.normal(0.0, np.sqrt(2.0 / (9 * ci)), size=(co, 9, ci)), np.zeros(co))
    params["head"] = (rng.normal(0.0, np.sqrt(1.0 / LEVELS[0]), size=(OUT_CH, LEVELS[0])), np.zeros(OUT_CH))
    return params
