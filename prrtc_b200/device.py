"""Device-side views of collision contexts and small torch helpers.

torch provides device memory and streams; the computation itself is in
libprrtc_b200.so.  A ``DeviceContext`` holds the collision_context tensors of
one robot + world on a CUDA device and fills the C structs of the C-ABI.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib

ROBOT_SPEC = {
    "fk_twists": (torch.float32, 6), "fk_parent_tf": (torch.float32, 7),
    "fk_parent_idx": (torch.int32, 0), "fk_act_idx": (torch.int32, 0),
    "fk_mimic_mul": (torch.float32, 0), "fk_mimic_off": (torch.float32, 0),
    "fk_mimic_act_idx": (torch.int32, 0), "fk_topo_inv": (torch.int32, 0),
    "sphere_link_idx": (torch.int32, 0), "sphere_local": (torch.float32, 3),
    "sphere_radius": (torch.float32, 0),
    "coarse_sphere_link_idx": (torch.int32, 0), "coarse_sphere_local": (torch.float32, 3),
    "coarse_sphere_radius": (torch.float32, 0), "fine_link_offsets": (torch.int32, 0),
    "coarse_self_pairs": (torch.int32, 2), "self_pair_ranges": (torch.int32, 2),
}
WORLD_SPEC = {
    "world_spheres": (torch.float32, 4), "world_capsules": (torch.float32, 7),
    "world_boxes": (torch.float32, 15), "world_halfspaces": (torch.float32, 6),
    "self_pairs": (torch.int32, 2),
}
REQUIRED_KEYS = (
    "fk_twists", "fk_parent_tf", "fk_parent_idx", "fk_act_idx", "fk_mimic_mul", "fk_mimic_off",
    "fk_mimic_act_idx", "fk_topo_inv", "sphere_link_idx", "sphere_local", "sphere_radius",
)


def cuda_device(device=None) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("prrtc_b200 requires a CUDA device (sm_100a); none is available")
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise ValueError(f"prrtc_b200 runs on CUDA devices only, got {d}")
    return d


# host->device bytes copied by this module (as_tensor of host data, upload);
# read and reset by callers that account for their transfers
H2D_BYTES = [0]


def as_tensor(x, dtype: torch.dtype, device: torch.device, cols: int = 0) -> torch.Tensor:
    """Contiguous tensor of `dtype` on `device`; `cols` > 0 reshapes to (-1, cols)."""
    if isinstance(x, torch.Tensor):
        if x.device != device and device.type == "cuda":
            H2D_BYTES[0] += x.numel() * torch.empty((), dtype=dtype).element_size()
        t = x.to(device=device, dtype=dtype)
    else:
        t = torch.as_tensor(np.asarray(x), dtype=dtype)
        if device.type == "cuda":
            H2D_BYTES[0] += t.numel() * t.element_size()
        t = t.to(device)
    if cols:
        t = t.reshape(-1, cols)
    return t.contiguous()


def upload(arrays, device: torch.device) -> list[torch.Tensor]:
    """Host arrays -> device tensors through ONE pinned staging buffer and one
    host-to-device copy (each array 256-byte aligned inside it)."""
    st = Stager(device)
    keys = [st.add(a, _TORCH_DTYPE[np.asarray(a).dtype.str[1:]]) for a in arrays]
    st.commit()
    return [st.get(k) for k in keys]


_TORCH_DTYPE = {"f4": torch.float32, "i4": torch.int32, "u1": torch.uint8, "i8": torch.int64, "f8": torch.float64}
_NUMPY_DTYPE = {torch.float32: np.float32, torch.int32: np.int32, torch.uint8: np.uint8, torch.int64: np.int64,
                torch.float64: np.float64}


class Stager:
    """Inputs of one call gathered for a single pinned host->device copy.

    ``add`` queues a host array (numpy, list, CPU tensor) and returns a key;
    a tensor already on the device passes through without a copy.
    ``reserve`` sets aside a region that ``on_fill`` callbacks write straight
    into the pinned buffer.  After ``commit`` (one host->device copy),
    ``get(key)`` is the device tensor."""

    def __init__(self, device: torch.device):
        self.device = device
        self._host: list = []  # np.ndarray, or (nbytes, torch dtype, shape) for a reserved region
        self._fill: list = []
        self._offsets: list[int] = []
        self._dev: list[torch.Tensor] | None = None

    def add(self, x, dtype: torch.dtype, shape=None):
        if isinstance(x, torch.Tensor) and x.device == self.device:
            t = x.to(dtype=dtype)
            return ("t", (t.reshape(shape) if shape is not None else t).contiguous())
        a = np.asarray(x.cpu() if isinstance(x, torch.Tensor) else x, dtype=_NUMPY_DTYPE[dtype])
        if shape is not None:
            a = a.reshape(shape)
        self._host.append(np.ascontiguousarray(a))
        return ("h", len(self._host) - 1)

    def reserve(self, dtype: torch.dtype, shape):
        n = int(np.prod(shape)) * torch.empty((), dtype=dtype).element_size()
        self._host.append((n, dtype, tuple(shape)))
        return ("h", len(self._host) - 1)

    def on_fill(self, fn) -> None:
        """fn(host_bytes: np.ndarray[uint8], offset_of: callable(key) -> int)."""
        self._fill.append(fn)

    def commit(self) -> None:
        offs, total = [], 0
        for a in self._host:
            offs.append(total)
            n = a.nbytes if isinstance(a, np.ndarray) else a[0]
            total += (n + 255) & ~255
        total = max(total, 256)
        host = torch.empty(total, dtype=torch.uint8, pin_memory=True)
        hv = host.numpy()
        for a, o in zip(self._host, offs):
            if isinstance(a, np.ndarray):
                hv[o:o + a.nbytes] = a.reshape(-1).view(np.uint8)
        self._offsets = offs
        for fn in self._fill:
            fn(hv, lambda key: offs[key[1]])
        dev = torch.empty(total, dtype=torch.uint8, device=self.device)
        H2D_BYTES[0] += total
        # torch's caching host allocator records the copy on the stream and keeps
        # the pinned block out of reuse until that copy has run
        dev.copy_(host, non_blocking=True)
        out = []
        for a, o in zip(self._host, offs):
            if isinstance(a, np.ndarray):
                out.append(dev[o:o + a.nbytes].view(_TORCH_DTYPE[a.dtype.str[1:]]).reshape(a.shape))
            else:
                out.append(dev[o:o + a[0]].view(a[1]).reshape(a[2]))
        self._dev = out

    def get(self, key) -> torch.Tensor:
        kind, v = key
        return v if kind == "t" else self._dev[v]


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None or t.numel() == 0:
        return None
    return t.data_ptr()


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


class DeviceContext:
    """collision_context tensors on one CUDA device."""

    def __init__(self, ctx: dict | None, device: torch.device, world_keys: bool = True, stager: Stager | None = None):
        """With a ``stager``, host tables are queued on it and the tensors exist
        after ``finish()`` (called once the stager has committed)."""
        self.device = device
        self.t: dict[str, torch.Tensor] = {}
        self._keys: dict = {}
        spec = dict(ROBOT_SPEC)
        if world_keys:
            spec.update(WORLD_SPEC)
        for k, (dt, cols) in spec.items():
            if ctx is not None and k in ctx and ctx[k] is not None:
                if stager is not None:
                    self._keys[k] = stager.add(ctx[k], dt, (-1, cols) if cols else (-1,))
                else:
                    self.t[k] = as_tensor(ctx[k], dt, device, cols)
            else:
                self.t[k] = torch.zeros((0, cols) if cols else (0,), dtype=dt, device=device)
        self._stager = stager

    def finish(self) -> "DeviceContext":
        for k, key in self._keys.items():
            self.t[k] = self._stager.get(key)
        self._keys, self._stager = {}, None
        return self

    def n(self, key: str) -> int:
        return int(self.t[key].shape[0])

    def robot(self) -> _lib.Robot:
        t = self.t
        r = _lib.Robot()
        for k in ("fk_twists", "fk_parent_tf", "fk_parent_idx", "fk_act_idx", "fk_mimic_mul", "fk_mimic_off",
                  "fk_mimic_act_idx", "fk_topo_inv", "sphere_link_idx", "sphere_local", "sphere_radius",
                  "coarse_sphere_link_idx", "coarse_sphere_local", "coarse_sphere_radius", "fine_link_offsets",
                  "coarse_self_pairs", "self_pair_ranges"):
            setattr(r, k, ptr(t[k]))
        r.n_joints = self.n("fk_parent_idx")
        r.n_spheres = self.n("sphere_link_idx")
        nk = self.n("coarse_sphere_link_idx")
        # the coarse model needs its K+1 fine offsets; otherwise it is absent
        r.n_coarse = nk if self.n("fine_link_offsets") >= nk + 1 else 0
        r.n_coarse_self_pairs = min(self.n("coarse_self_pairs"), self.n("self_pair_ranges")) if r.n_coarse else 0
        return r

    def world(self) -> _lib.World:
        t = self.t
        w = _lib.World()
        for k in ("world_spheres", "world_capsules", "world_boxes", "world_halfspaces", "self_pairs"):
            setattr(w, k, ptr(t[k]))
        w.n_world_spheres = self.n("world_spheres")
        w.n_world_capsules = self.n("world_capsules")
        w.n_world_boxes = self.n("world_boxes")
        w.n_world_halfspaces = self.n("world_halfspaces")
        w.n_self_pairs = self.n("self_pairs")
        return w


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    # torch's CUDA allocator returns 512-byte aligned blocks
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def byref(s):
    return C.byref(s)
