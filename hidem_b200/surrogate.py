"""Learned warm start: the settling surrogate (``hidem_surrogate_*``).

A coordinate MLP maps normalised inputs per particle (by default 5: x, y, z, local ice
thickness and bed height under the particle; ``config.inputs`` of them in general, e.g.
the lattice-neighbourhood inputs of ``hidem_b200.settle.lattice_inputs``) to its settled
displacement (3 components, normalised).
Training and inference run in the library's own kernels: BF16 tensor-core GEMMs for the
hidden layers, CUDA-core kernels for the output layer, loss, reductions and Adam. No
counterpart in the reference, which settles every geometry from rest; the plain settling
run still decides when a warm-started geometry has settled (see ``hidem_b200.settle``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

N_IN = 5      # default inputs per row
N_OUT = 3
N_FEAT = 128  # first-layer width of the default inputs


def feature_width(nin: int, bands: int) -> int:
    """First layer's input width: nin * (1 + 2 bands) rounded up to a multiple of 128."""
    return max(128, -(-nin * (1 + 2 * bands) // 128) * 128)


def default_config(**over) -> abi.HidemSurrogateConfig:
    lib = abi.load()
    c = abi.HidemSurrogateConfig()
    lib.hidem_surrogate_config_default(C.byref(c))
    for k, v in over.items():
        setattr(c, k, v)
    return c


def param_shapes(cfg: abi.HidemSurrogateConfig) -> list[tuple[str, tuple[int, ...]]]:
    """Names and shapes of the parameters in the library's flat order."""
    out = []
    k = feature_width(cfg.inputs, cfg.fourier_bands)
    for l in range(cfg.hidden_layers):
        out.append((f"W{l}", (cfg.width, k)))
        out.append((f"b{l}", (cfg.width,)))
        k = cfg.width
    out.append(("Wo", (N_OUT, cfg.width)))
    out.append(("bo", (N_OUT,)))
    return out


def unflatten(flat: np.ndarray, cfg) -> dict:
    out, o = {}, 0
    for name, shp in param_shapes(cfg):
        n = int(np.prod(shp))
        out[name] = flat[o:o + n].reshape(shp)
        o += n
    return out


def flatten(params: dict, cfg) -> np.ndarray:
    return np.concatenate([np.asarray(params[n], np.float32).ravel() for n, _ in param_shapes(cfg)])


class Surrogate:
    def __init__(self, cfg: abi.HidemSurrogateConfig | None = None, device: int = 0):
        self._lib = abi.load()
        self.cfg = cfg if cfg is not None else default_config()
        h = C.c_void_p()
        st = self._lib.hidem_surrogate_create(C.byref(self.cfg), int(device), C.byref(h))
        if st != abi.HIDEM_OK:
            raise abi.HidemError(st, self._lib.hidem_create_error().decode())
        self._s = h
        self.num_params = int(self._lib.hidem_surrogate_num_params(h))

    def _check(self, st: int) -> None:
        if st != abi.HIDEM_OK:
            raise abi.HidemError(st, self._lib.hidem_surrogate_last_error(self._s).decode())

    @staticmethod
    def _f32(a, cols):
        a = np.ascontiguousarray(a, dtype=np.float32)
        assert a.ndim == 2 and a.shape[1] == cols
        return a

    def get_params(self) -> np.ndarray:
        out = np.empty(self.num_params, np.float32)
        self._check(self._lib.hidem_surrogate_get_params(self._s, out.ctypes.data))
        return out

    def set_params(self, flat: np.ndarray) -> None:
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        assert flat.shape == (self.num_params,)
        self._check(self._lib.hidem_surrogate_set_params(self._s, flat.ctypes.data))

    def set_data(self, inputs, targets) -> None:
        x, t = self._f32(inputs, self.cfg.inputs), self._f32(targets, N_OUT)
        self._check(self._lib.hidem_surrogate_set_data(self._s, x.ctypes.data, t.ctypes.data, x.shape[0]))

    def train(self, steps: int) -> float:
        loss = C.c_double()
        self._check(self._lib.hidem_surrogate_train(self._s, int(steps), C.byref(loss)))
        return loss.value

    def predict(self, inputs) -> np.ndarray:
        x = self._f32(inputs, self.cfg.inputs)
        out = np.empty((x.shape[0], N_OUT), np.float32)
        self._check(self._lib.hidem_surrogate_predict(self._s, x.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    def predict_device(self, inputs_ptr: int, n: int, out_ptr: int) -> None:
        """Predictions for n rows already in device memory (device pointers to [n][inputs]
        and [n][3] FP32 arrays, e.g. torch tensors' data_ptr())."""
        self._check(self._lib.hidem_surrogate_predict_device(self._s, inputs_ptr, int(n), out_ptr))

    def set_forward(self, kind: int) -> None:
        """The forward pass's kernel: abi.SURROGATE_FORWARD_AUTO, _BLOCK or _PINGPONG."""
        self._check(self._lib.hidem_surrogate_set_forward(self._s, int(kind)))

    @property
    def stream_handle(self) -> int:
        """The cudaStream_t the surrogate's work runs on."""
        return int(self._lib.hidem_surrogate_get_stream(self._s) or 0)

    def gradients(self, inputs, targets) -> tuple[np.ndarray, float]:
        x, t = self._f32(inputs, self.cfg.inputs), self._f32(targets, N_OUT)
        g = np.empty(self.num_params, np.float32)
        loss = C.c_double()
        self._check(self._lib.hidem_surrogate_gradients(self._s, x.ctypes.data, t.ctypes.data, x.shape[0],
                                                        g.ctypes.data, C.byref(loss)))
        return g, loss.value

    def close(self) -> None:
        if getattr(self, "_s", None):
            self._lib.hidem_surrogate_destroy(self._s)
            self._s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _main(argv=None) -> None:
    """python -m hidem_b200.surrogate [--rows N] [--repeat R]: forward throughput of the
    default network on N random rows (the tensor-core GEMMs and their epilogues)."""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=1 << 20)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--inputs", type=int, default=N_IN)
    ap.add_argument("--bands", type=int, default=8)
    a = ap.parse_args(argv)
    cfg = default_config(inputs=a.inputs, fourier_bands=a.bands)
    u = np.random.default_rng(0).uniform(-1, 1, (a.rows, a.inputs)).astype(np.float32)
    import torch
    with Surrogate(cfg) as net:
        net.predict(u[: min(a.rows, 16384)])
        best = float("inf")
        for _ in range(a.repeat):
            t0 = time.perf_counter()
            net.predict(u)
            best = min(best, time.perf_counter() - t0)
        # inputs resident in device memory: features + fused network only, CUDA events on
        # the surrogate's stream
        du = torch.from_numpy(u).cuda()
        dy = torch.empty((a.rows, N_OUT), dtype=torch.float32, device="cuda")
        stream = torch.cuda.ExternalStream(net.stream_handle)
        dev = float("inf")
        for _ in range(a.repeat + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            net.predict_device(du.data_ptr(), a.rows, dy.data_ptr())
            e1.record(stream)
            torch.cuda.synchronize()
            dev = min(dev, e0.elapsed_time(e1) / 1e3)
    k0 = feature_width(cfg.inputs, cfg.fourier_bands)
    flops = 2.0 * a.rows * (k0 * cfg.width + (cfg.hidden_layers - 1) * cfg.width ** 2 + N_OUT * cfg.width)
    print(json.dumps({"rows": a.rows, "seconds": best, "tflops": flops / best / 1e12,
                      "device_seconds": dev, "device_tflops": flops / dev / 1e12}))


if __name__ == "__main__":
    _main()
