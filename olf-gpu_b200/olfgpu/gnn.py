"""Learned warm start: a message-passing graph network predicting each scenario's per-bus (dVm, dVa) from the base case.

Model (hidden width H = 64, 4 layers, BF16 weights and activations, FP32 accumulation), per sample over the bus graph:

    h0      = relu(X0 . Win + bin)                              X0: base-case [Vm, Va, P, Q, PQ?, PV?, slack?] and the
                                                                outaged branch's endpoint flag and base P, Q flow
    P, Q    = h . Wsrc, h . Wdst                                (one [H x 2H] GEMM)
    agg_i   = sum over directed edges e = (j -> i), e not in the outaged branch, of relu(P_j + Q_i + Es_e . We + bmsg)
    h      <- h + relu([h | agg] . Wupd + bupd)                 (residual)
    out     = h . Wout + bout                                   (the first two columns: normalised dVm, dVa)

Es_e are the branch's (r, x, b, ratio), normalised.  Every kernel is the library's (``olfgpu_gnn_*`` in
``include/olfgpu_b200.h``); PyTorch only owns the device memory and the data loading.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Dict, List, Optional

import numpy as np

from . import native

H = 64
FEAT_IN = 16          # 10 input features (7 per bus, 3 of the scenario's outage) padded to the 16-column MMA tile
FEAT_OUT = 16         # 2 outputs padded to 16 columns


def _lib():
    L = native.load()
    if not hasattr(L, "_gnn_ready"):
        vp = ctypes.c_void_p
        i = ctypes.c_int
        f = ctypes.c_float
        L.olfgpu_gnn_last_error.restype = ctypes.c_char_p
        sig = {
            "olfgpu_gnn_gemm": [i, i, i, i, vp, vp, vp, vp, i, vp, vp, vp, i, vp, vp],
            "olfgpu_gnn_tc_timeouts": [vp],
            "olfgpu_gnn_gemm_dw": [i, i, i, i, vp, vp, vp, vp, vp, vp, i, vp],
            "olfgpu_gnn_message_forward": [i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp],
            "olfgpu_gnn_message_backward": [i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp],
            "olfgpu_gnn_edge_project": [i, vp, vp, vp, vp],
            "olfgpu_gnn_edge_project_backward": [i, vp, vp, vp, vp, vp],
            "olfgpu_gnn_relu_grad": [ctypes.c_longlong, i, i, vp, vp, vp, vp, vp],
            "olfgpu_gnn_adam": [i, i, i, vp, vp, vp, vp, f, f, f, f, i, vp, vp, vp],
            "olfgpu_gnn_mse": [i, i, vp, vp, vp, vp, vp],
            "olfgpu_gnn_copy_cols": [i, i, vp, i, i, vp, i, i, i, vp],
            "olfgpu_gnn_compose_start": [i, i, vp, i, ctypes.c_double, ctypes.c_double, vp, vp, vp, vp, vp],
            "olfgpu_gnn_message_forward_compact": [i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp],
            "olfgpu_gnn_compact_inputs": [i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp],
            "olfgpu_gnn_compose_start_compact": [i, i, vp, vp, i, i, vp, vp, ctypes.c_double, ctypes.c_double, vp, vp,
                                                 vp, vp, vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L._gnn_ready = True
    return L


def _call(name, *args):
    L = _lib()
    rc = getattr(L, name)(*args)
    if rc != 0:
        raise native.NativeError(f"{name}: {L.olfgpu_gnn_last_error().decode()}")


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def tc_timeouts() -> int:
    """Tensor-core GEMM tiles that gave up waiting for their MMAs since the library was loaded (0 on a working GPU)."""
    v = ctypes.c_int(0)
    _call("olfgpu_gnn_tc_timeouts", ctypes.byref(v))
    return v.value


def gemm(a1, a2, w, bias=None, relu=False, residual=None, out_f32=False, save_z=False):
    """Y = [a1 | a2] . w (+ bias), z = relu(Y) or Y, out = z (+ residual), on the tensor cores; BF16 CUDA tensors in.
    Returns (out, z or None): out BF16 [M, N] (FP32 with out_f32)."""
    import torch
    M, K1 = a1.shape
    K2 = 0 if a2 is None else a2.shape[1]
    N = w.shape[1]
    out = torch.empty((M, N), dtype=torch.float32 if out_f32 else torch.bfloat16, device=a1.device)
    z = torch.empty((M, N), dtype=torch.bfloat16, device=a1.device) if save_z else None
    _call("olfgpu_gnn_gemm", M, K1, K2, N, _ptr(a1), _ptr(a2), _ptr(w), _ptr(bias), 1 if relu else 0, _ptr(residual),
          None if out_f32 else _ptr(out), _ptr(out) if out_f32 else None, N, _ptr(z), _stream())
    return out, z


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@dataclasses.dataclass
class GraphData:
    """Directed edges (both directions of every closed branch) with destination- and source-ordered lists."""
    nb: int
    n_edges: int
    src: "object"
    dst: "object"
    branch: "object"
    in_ptr: "object"
    in_edge: "object"
    out_ptr: "object"
    out_edge: "object"
    es: "object"        # [n_edges, 4] float32 normalised (r, x, b, ratio)

    @staticmethod
    def from_grid(g, device="cuda"):
        import torch
        nbr = g.f.shape[0]
        src = np.concatenate([g.f, g.t]).astype(np.int32)
        dst = np.concatenate([g.t, g.f]).astype(np.int32)
        branch = np.concatenate([np.arange(nbr), np.arange(nbr)]).astype(np.int32)
        feats = np.stack([g.r, g.x, g.b, g.ratio], axis=1)
        feats = (feats - feats.mean(0)) / np.maximum(feats.std(0), 1e-9)
        es = np.concatenate([feats, feats]).astype(np.float32)
        order_in = np.argsort(dst, kind="stable")
        order_out = np.argsort(src, kind="stable")
        in_ptr = np.zeros(g.n_bus + 1, np.int32)
        np.add.at(in_ptr, dst + 1, 1)
        in_ptr = np.cumsum(in_ptr).astype(np.int32)
        out_ptr = np.zeros(g.n_bus + 1, np.int32)
        np.add.at(out_ptr, src + 1, 1)
        out_ptr = np.cumsum(out_ptr).astype(np.int32)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        return GraphData(g.n_bus, 2 * nbr, t(src), t(dst), t(branch), t(in_ptr), t(order_in.astype(np.int32)),
                         t(out_ptr), t(order_out.astype(np.int32)), t(es))


# Parameter shapes: name -> (K, N) of a [K x N] matrix (vectors have K = 1)
def param_shapes(layers: int) -> Dict[str, tuple]:
    shapes = {"w_in": (FEAT_IN, H), "b_in": (1, H)}
    for l in range(layers):
        shapes[f"w_pq{l}"] = (H, 2 * H)
        shapes[f"w_e{l}"] = (4, H)
        shapes[f"b_msg{l}"] = (1, H)
        shapes[f"w_upd{l}"] = (2 * H, H)
        shapes[f"b_upd{l}"] = (1, H)
    shapes["w_out"] = (H, FEAT_OUT)
    shapes["b_out"] = (1, FEAT_OUT)
    return shapes


def init_params(layers: int, seed: int) -> Dict[str, np.ndarray]:
    rng = np.random.default_rng(seed)
    p = {}
    for name, (k, n) in param_shapes(layers).items():
        if name.startswith("b_"):
            p[name] = np.zeros((k, n), np.float32)
        elif name == "w_out":
            w = np.zeros((k, n), np.float32)
            w[:, :2] = rng.normal(0, 0.1 / np.sqrt(k), (k, 2))
            p[name] = w
        elif name == "w_in":
            w = rng.normal(0, np.sqrt(2.0 / 10), (k, n)).astype(np.float32)
            w[10:] = 0.0                                     # 10 input features, the tile padding stays zero
            p[name] = w
        elif name.startswith("w_upd"):
            p[name] = (rng.normal(0, np.sqrt(2.0 / k), (k, n)) * 0.5).astype(np.float32)
        else:
            p[name] = rng.normal(0, np.sqrt(2.0 / k), (k, n)).astype(np.float32)
    return p


class WarmStartNet:
    """The network on the device: FP32 master weights, BF16 copies (and transposes) for the kernels, Adam state."""

    def __init__(self, graph: GraphData, layers: int = 4, seed: int = 0, params: Optional[Dict] = None):
        import torch
        self.graph = graph
        self.layers = layers
        self.dev = torch.device("cuda")
        host = params if params is not None else init_params(layers, seed)
        self.w = {k: torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(self.dev) for k, v in host.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.step = 0
        self.wb, self.wt = {}, {}
        for k, v in self.w.items():
            if k.startswith("w_") and not k.startswith("w_e"):
                kk, nn = v.shape
                self.wb[k] = v.to(torch.bfloat16).contiguous()
                rows = 16 if k == "w_out" else nn
                t = torch.zeros((rows, kk), dtype=torch.bfloat16, device=self.dev)
                t[:nn] = v.t().to(torch.bfloat16)
                self.wt[k] = t
        self._partial = None

    # ------------------------------------------------------------------------------------------------------------
    def forward_rows(self, x0, outage, rows=None, base_pq=None, keep_pq: bool = False):
        """Inference only.  rows None: every bus of every sample (x0 [B * nb, 16]), returning (out, per-layer PQ when
        keep_pq).  rows = (row_node, row_sample, row_of) device int32 tensors: x0 holds only those rows [R, 16] and a
        neighbour outside them reads base_pq[l] (the outage-free sample's layer-l PQ, [nb, 128]).  Same arithmetic per
        row either way."""
        import torch
        g = self.graph
        M = x0.shape[0]
        B = outage.shape[0]
        st = _stream()
        bf = torch.bfloat16
        h = torch.empty((M, H), dtype=bf, device=self.dev)
        _call("olfgpu_gnn_gemm", M, FEAT_IN, 0, H, _ptr(x0), None, _ptr(self.wb["w_in"]), _ptr(self.w["b_in"]), 1,
              None, _ptr(h), None, H, None, st)
        pqs = []
        for l in range(self.layers):
            c = torch.empty((g.n_edges, H), dtype=torch.float32, device=self.dev)
            _call("olfgpu_gnn_edge_project", g.n_edges, _ptr(g.es), _ptr(self.w[f"w_e{l}"]), _ptr(c), st)
            pq = torch.empty((M, 2 * H), dtype=bf, device=self.dev)
            _call("olfgpu_gnn_gemm", M, H, 0, 2 * H, _ptr(h), None, _ptr(self.wb[f"w_pq{l}"]), None, 0, None, _ptr(pq),
                  None, 2 * H, None, st)
            agg = torch.empty((M, H), dtype=bf, device=self.dev)
            if rows is None:
                _call("olfgpu_gnn_message_forward", B, g.nb, _ptr(g.in_ptr), _ptr(g.in_edge), _ptr(g.src),
                      _ptr(g.branch), _ptr(outage), _ptr(pq), _ptr(c), _ptr(self.w[f"b_msg{l}"]), _ptr(agg), st)
            else:
                rn, rs, ro = rows
                _call("olfgpu_gnn_message_forward_compact", M, g.nb, _ptr(rn), _ptr(rs), _ptr(ro), _ptr(g.in_ptr),
                      _ptr(g.in_edge), _ptr(g.src), _ptr(g.branch), _ptr(outage), _ptr(pq), _ptr(base_pq[l]), _ptr(c),
                      _ptr(self.w[f"b_msg{l}"]), _ptr(agg), st)
            if keep_pq:
                pqs.append(pq)
            hn = torch.empty((M, H), dtype=bf, device=self.dev)
            _call("olfgpu_gnn_gemm", M, H, H, H, _ptr(h), _ptr(agg), _ptr(self.wb[f"w_upd{l}"]),
                  _ptr(self.w[f"b_upd{l}"]), 1, _ptr(h), _ptr(hn), None, H, None, st)
            h = hn
        out = torch.empty((M, FEAT_OUT), dtype=torch.float32, device=self.dev)
        _call("olfgpu_gnn_gemm", M, H, 0, FEAT_OUT, _ptr(h), None, _ptr(self.wb["w_out"]), _ptr(self.w["b_out"]), 0,
              None, None, _ptr(out), FEAT_OUT, None, st)
        return (out, pqs) if keep_pq else out

    def forward(self, x0, outage, keep: bool = False):
        """x0: [B * nb, 16] bf16, outage: [B] int32 (closed-branch index per sample). Returns out [B * nb, 16] fp32."""
        import torch
        g = self.graph
        M = x0.shape[0]
        B = outage.shape[0]
        st = _stream()
        bf = torch.bfloat16
        h = torch.empty((M, H), dtype=bf, device=self.dev)
        _call("olfgpu_gnn_gemm", M, FEAT_IN, 0, H, _ptr(x0), None, _ptr(self.wb["w_in"]), _ptr(self.w["b_in"]), 1,
              None, _ptr(h), None, H, None, st)
        saved = {"x0": x0, "h": [h], "pq": [], "agg": [], "z": [], "c": []}
        for l in range(self.layers):
            c = torch.empty((g.n_edges, H), dtype=torch.float32, device=self.dev)
            _call("olfgpu_gnn_edge_project", g.n_edges, _ptr(g.es), _ptr(self.w[f"w_e{l}"]), _ptr(c), st)
            pq = torch.empty((M, 2 * H), dtype=bf, device=self.dev)
            _call("olfgpu_gnn_gemm", M, H, 0, 2 * H, _ptr(h), None, _ptr(self.wb[f"w_pq{l}"]), None, 0, None, _ptr(pq),
                  None, 2 * H, None, st)
            agg = torch.empty((M, H), dtype=bf, device=self.dev)
            _call("olfgpu_gnn_message_forward", B, g.nb, _ptr(g.in_ptr), _ptr(g.in_edge), _ptr(g.src), _ptr(g.branch),
                  _ptr(outage), _ptr(pq), _ptr(c), _ptr(self.w[f"b_msg{l}"]), _ptr(agg), st)
            z = torch.empty((M, H), dtype=bf, device=self.dev) if keep else None
            hn = torch.empty((M, H), dtype=bf, device=self.dev)
            _call("olfgpu_gnn_gemm", M, H, H, H, _ptr(h), _ptr(agg), _ptr(self.wb[f"w_upd{l}"]),
                  _ptr(self.w[f"b_upd{l}"]), 1, _ptr(h), _ptr(hn), None, H, _ptr(z), st)
            if keep:
                saved["pq"].append(pq)
                saved["agg"].append(agg)
                saved["z"].append(z)
                saved["c"].append(c)
                saved["h"].append(hn)
            h = hn
        out = torch.empty((M, FEAT_OUT), dtype=torch.float32, device=self.dev)
        _call("olfgpu_gnn_gemm", M, H, 0, FEAT_OUT, _ptr(h), None, _ptr(self.wb["w_out"]), _ptr(self.w["b_out"]), 0,
              None, None, _ptr(out), FEAT_OUT, None, st)
        if keep:
            saved["h_last"] = h
            saved["outage"] = outage
            self._saved = saved
        return out

    def _dw(self, M, k1, k2, n, a1, a2, dz, name_w, name_b):
        import torch
        chunks = 296
        need = chunks * ((k1 + k2) * n + n)
        if self._partial is None or self._partial.numel() < need:
            self._partial = torch.empty(need, dtype=torch.float32, device=self.dev)
        gw = torch.empty(((k1 + k2), n), dtype=torch.float32, device=self.dev)
        gb = torch.empty((1, n), dtype=torch.float32, device=self.dev) if name_b else None
        _call("olfgpu_gnn_gemm_dw", M, k1, k2, n, _ptr(a1), _ptr(a2), _ptr(dz), _ptr(gw), _ptr(gb),
              _ptr(self._partial), chunks, _stream())
        self.grad[name_w] = gw
        if name_b:
            self.grad[name_b] = gb

    def backward(self, d_out):
        """d_out: [M, 16] fp32 gradient of the loss w.r.t. the output. Fills self.grad (fp32 per parameter)."""
        import torch
        s = self._saved
        g = self.graph
        M = d_out.shape[0]
        B = s["outage"].shape[0]
        st = _stream()
        bf = torch.bfloat16
        self.grad = {}
        dzo = torch.empty((M, FEAT_OUT), dtype=bf, device=self.dev)
        _call("olfgpu_gnn_relu_grad", M * FEAT_OUT, FEAT_OUT, FEAT_OUT, _ptr(d_out), None, _ptr(dzo), None, st)
        self._dw(M, H, 0, FEAT_OUT, s["h_last"], None, dzo, "w_out", "b_out")
        dh = torch.empty((M, H), dtype=torch.float32, device=self.dev)
        _call("olfgpu_gnn_gemm", M, FEAT_OUT, 0, H, _ptr(dzo), None, _ptr(self.wt["w_out"]), None, 0, None, None,
              _ptr(dh), H, None, st)
        tmp2 = torch.empty((M, 2 * H), dtype=torch.float32, device=self.dev)
        tmp = torch.empty((M, H), dtype=torch.float32, device=self.dev)
        dagg = torch.empty((M, H), dtype=torch.float32, device=self.dev)
        for l in reversed(range(self.layers)):
            h_l, agg, pq, z, c = s["h"][l], s["agg"][l], s["pq"][l], s["z"][l], s["c"][l]
            dz = torch.empty((M, H), dtype=bf, device=self.dev)
            _call("olfgpu_gnn_relu_grad", M * H, H, H, _ptr(dh), _ptr(z), _ptr(dz), None, st)
            self._dw(M, H, H, H, h_l, agg, dz, f"w_upd{l}", f"b_upd{l}")
            _call("olfgpu_gnn_gemm", M, H, 0, 2 * H, _ptr(dz), None, _ptr(self.wt[f"w_upd{l}"]), None, 0, None, None,
                  _ptr(tmp2), 2 * H, None, st)
            # residual: dh stays; the [h | agg] halves of the update's input gradient split off
            _call("olfgpu_gnn_copy_cols", M, H, _ptr(tmp2), 2 * H, 0, _ptr(dh), H, 0, 1, st)
            _call("olfgpu_gnn_copy_cols", M, H, _ptr(tmp2), 2 * H, H, _ptr(dagg), H, 0, 0, st)
            dpq = torch.empty((M, 2 * H), dtype=torch.float32, device=self.dev)
            dc = torch.empty((g.n_edges, H), dtype=torch.float32, device=self.dev)
            _call("olfgpu_gnn_message_backward", B, g.nb, g.n_edges, _ptr(g.in_ptr), _ptr(g.in_edge), _ptr(g.out_ptr),
                  _ptr(g.out_edge), _ptr(g.src), _ptr(g.dst), _ptr(g.branch), _ptr(s["outage"]), _ptr(pq), _ptr(c),
                  _ptr(self.w[f"b_msg{l}"]), _ptr(dagg), _ptr(dpq), _ptr(dc), st)
            gwe = torch.empty((4, H), dtype=torch.float32, device=self.dev)
            gbm = torch.empty((1, H), dtype=torch.float32, device=self.dev)
            _call("olfgpu_gnn_edge_project_backward", g.n_edges, _ptr(g.es), _ptr(dc), _ptr(gwe), _ptr(gbm), st)
            self.grad[f"w_e{l}"] = gwe
            self.grad[f"b_msg{l}"] = gbm
            dpqb = torch.empty((M, 2 * H), dtype=bf, device=self.dev)
            _call("olfgpu_gnn_relu_grad", M * 2 * H, 2 * H, 2 * H, _ptr(dpq), None, _ptr(dpqb), None, st)
            self._dw(M, H, 0, 2 * H, h_l, None, dpqb, f"w_pq{l}", None)
            _call("olfgpu_gnn_gemm", M, 2 * H, 0, H, _ptr(dpqb), None, _ptr(self.wt[f"w_pq{l}"]), None, 0, None, None,
                  _ptr(tmp), H, None, st)
            _call("olfgpu_gnn_copy_cols", M, H, _ptr(tmp), H, 0, _ptr(dh), H, 0, 1, st)
        dz0 = torch.empty((M, H), dtype=bf, device=self.dev)
        _call("olfgpu_gnn_relu_grad", M * H, H, H, _ptr(dh), _ptr(s["h"][0]), _ptr(dz0), None, st)
        self._dw(M, FEAT_IN, 0, H, s["x0"], None, dz0, "w_in", "b_in")
        return self.grad

    def loss_and_grad(self, x0, outage, target):
        """MSE of the first two output columns against target [M, 2] fp32; backward included. Returns the loss."""
        import torch
        out = self.forward(x0, outage, keep=True)
        M = out.shape[0]
        d_out = torch.empty_like(out)
        nblk = (M + 255) // 256
        partial = torch.empty(nblk, dtype=torch.float32, device=self.dev)
        _call("olfgpu_gnn_mse", M, FEAT_OUT, _ptr(out), _ptr(target), _ptr(d_out), _ptr(partial), _stream())
        self.backward(d_out)
        return float(partial.sum().item()) / (2 * M)

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        st = _stream()
        for k, w in self.w.items():
            kk, nn = w.shape
            _call("olfgpu_gnn_adam", w.numel(), kk, nn, _ptr(w), _ptr(self.grad[k]), _ptr(self.m[k]), _ptr(self.v[k]),
                  lr, beta1, beta2, eps, self.step, _ptr(self.wb.get(k)), _ptr(self.wt.get(k)), st)

    # ------------------------------------------------------------------------------------------------------------
    def state(self) -> Dict[str, np.ndarray]:
        out = {f"w.{k}": v.cpu().numpy() for k, v in self.w.items()}
        out.update({f"m.{k}": v.cpu().numpy() for k, v in self.m.items()})
        out.update({f"v.{k}": v.cpu().numpy() for k, v in self.v.items()})
        out["step"] = np.array(self.step)
        out["layers"] = np.array(self.layers)
        return out

    def save(self, path: str, extra: Optional[Dict[str, np.ndarray]] = None):
        d = self.state()
        if extra:
            d.update({f"x.{k}": v for k, v in extra.items()})
        tmp = path + ".tmp.npz"
        np.savez(tmp, **d)
        os.replace(tmp, path)

    @staticmethod
    def load(path: str, graph: GraphData):
        import torch
        d = np.load(path)
        layers = int(d["layers"])
        params = {k[2:]: d[k] for k in d.files if k.startswith("w.")}
        net = WarmStartNet(graph, layers, params=params)
        for k in net.w:
            net.m[k] = torch.from_numpy(d[f"m.{k}"]).to(net.dev)
            net.v[k] = torch.from_numpy(d[f"v.{k}"]).to(net.dev)
        net.step = int(d["step"])
        extra = {k[2:]: d[k] for k in d.files if k.startswith("x.")}
        return net, extra
