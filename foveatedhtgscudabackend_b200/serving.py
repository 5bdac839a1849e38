"""Request server over the C ABI's `fhtgs_server_*` entry points (include/fhtgs.h, "serving").

No counterpart in the reference, whose API renders one view or one stereo pair per blocking
call (`torch_bindings/rasterization.py:73-154`).  A `Server` keeps several scenes resident,
accepts stereo (or mono) view requests from any thread, and renders them by continuous
batching: whenever one of its frame slots is free, the oldest queued request and the other
queued requests of the same scene become one multi-view frame on that slot's stream, so
requests that arrive while others are on the GPU join the next frame of their scene, and the
frames of different slots overlap on the device.  Every frame's device memory is admitted
against an HBM budget.  A request's images are exactly the images `Renderer.render` (or the
drop-in `_C_stereo.render`) produces for the same views: batching changes the schedule, not a
pixel.

    srv = Server(device=0, hbm_budget_bytes=150e9)
    sid = srv.add_scene(*gaussians, K=8, active_sh_bases=16)
    t = srv.submit(sid, [left_view, right_view])          # scene.View or RasterizerSettings eyes
    for c in srv.poll(wait_ms=100):
        imgs = c.images                                   # torch tensors on the device
        srv.release(c.ticket)                             # server-owned outputs back to the pool
"""
from __future__ import annotations

import ctypes as C
import functools
import threading
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from . import scene as _scene
from .rasterization import BackgroundModel, RasterizerSettings, _check_gaussians, _Keep, _texture_size


class _DeviceArray:
    """`__cuda_array_interface__` of a server-owned output image (no copy)."""

    def __init__(self, ptr: int, shape: tuple[int, ...]):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4", "data": (ptr, False), "version": 3,
                                         "strides": None}


@dataclass
class Completion:
    ticket: int
    tag: int
    status: int
    frame_views: int
    submit_ms: float
    launch_ms: float
    done_ms: float
    message: str
    # torch tensors on the device: the caller's images, or views of server-owned output buffers
    # that stay valid until Server.release(ticket) or Server.close() (reading them later reads
    # freed device memory)
    images: list = field(default_factory=list)
    replica: int = 0     # ServerGroup: the replica that rendered it
    device: int = -1     # ServerGroup: the device its images lie on

    @property
    def ok(self) -> bool:
        return self.status == 0

    @property
    def latency_ms(self) -> float:
        return self.done_ms - self.submit_ms


@functools.lru_cache(maxsize=64)
def _all_visible_words(gw: int, gh: int) -> np.ndarray:
    return _scene.visibility_tables(gw, gh)[0]


def _eye_from(view, device: torch.device, keep: _Keep) -> _lib.Eye:
    """An fhtgs_eye from a scene.View (NumPy camera) or a RasterizerSettings (torch tensors)."""
    e = _lib.Eye()
    if isinstance(view, RasterizerSettings):
        M = view.M.detach().float().cpu().numpy().reshape(-1)
        VPM = view.VPM.detach().float().cpu().numpy().reshape(-1)
        VPR = view.VPR_inv.detach().float().cpu().numpy().reshape(-1)
        cam = view.cam_position.detach().float().cpu().numpy().reshape(-1)
        gaze = view.gaze_position.detach().float().cpu().numpy().reshape(-1)
        e.visibility_mask = keep.u32(view.visibility_mask, "visibility_mask")
        e.visibility_mask_area_table = keep.u32(view.visibility_mask_area_table, "visibility_mask_area_table")
        e.fovea_mask_area_table = keep.u32(view.fovea_mask_area_table, "fovea_mask_area_table")
    elif isinstance(view, _scene.View):
        M, VPM, VPR = view.M.reshape(-1), view.VPM.reshape(-1), view.VPR_inv.reshape(-1)
        cam, gaze = view.cam_position.reshape(-1), view.gaze_position.reshape(-1)
        gw, gh = view.grid_large
        if not np.array_equal(view.visibility_mask, _all_visible_words(gw, gh)):
            # a partial mask: its tables go to the device with the request
            def u(a):
                return torch.from_numpy(np.ascontiguousarray(a, np.uint32)).to(device)
            e.visibility_mask = keep.u32(u(view.visibility_mask), "visibility_mask")
            e.visibility_mask_area_table = keep.u32(u(view.visibility_mask_area_table), "visibility_mask_area_table")
    else:
        raise TypeError("an eye must be a scene.View or a RasterizerSettings")
    e.M[:] = [float(x) for x in M[:12]]
    e.VPM[:] = [float(x) for x in VPM[:16]]
    e.VPR_inv[:] = [float(x) for x in VPR[:16]]
    e.cam_position[:] = [float(x) for x in cam[:3]]
    e.gaze_x, e.gaze_y = float(gaze[0]), float(gaze[1])
    e.width, e.height = int(view.width), int(view.height)
    e.focal_x, e.focal_y = float(view.focal_x), float(view.focal_y)
    e.center_x, e.center_y = float(view.center_x), float(view.center_y)
    return e


def _scene_structs(device: torch.device, positions, scales, rotations, opacities, sh_0, sh_rest, *, K, active_sh_bases,
                   near_plane, far_plane, scale_modifier, to_chw, blur_periphery, aaa_mode, fast_math, background,
                   background_data, foveation, rings):
    """fhtgs_primitives and fhtgs_settings of a scene whose tensors lie on `device` (with the
    tensors they point into kept alive)."""
    if foveation not in _lib.FOVEATION:
        raise ValueError(f"foveation must be one of {sorted(_lib.FOVEATION)}")
    keep = _Keep(device)
    n, total_sh = _check_gaussians(positions, scales, rotations, opacities, sh_0, sh_rest)
    # the servers' streams do not wait for PyTorch's: the scene must be complete now
    torch.cuda.current_stream(device).synchronize()
    if scales.dtype == torch.float16:
        h, b = torch.float16, torch.bfloat16
        prims = _lib.Primitives(keep.f32(positions, "positions"), keep.typed(scales, "scales", h),
                                keep.typed(rotations, "rotations", h), keep.typed(opacities, "opacities", h),
                                keep.typed(sh_0, "sh_0", b), keep.typed(sh_rest, "sh_rest", b), n, total_sh,
                                _lib.STORAGE_HALF)
    else:
        prims = _lib.Primitives(keep.f32(positions, "positions"), keep.f32(scales, "scales"),
                                keep.f32(rotations, "rotations"), keep.f32(opacities, "opacities"),
                                keep.f32(sh_0, "sh_0"), keep.f32(sh_rest, "sh_rest"), n, total_sh,
                                _lib.STORAGE_FP32)
    if background_data is None:
        background_data = torch.zeros(1, device=device)
    bg_type = background.value
    tw, th = _texture_size(bg_type, background_data)
    st = _lib.Settings(int(K), int(active_sh_bases), float(near_plane), float(far_plane), float(scale_modifier),
                       int(bool(to_chw)), int(bool(blur_periphery)), int(bool(aaa_mode)), bg_type,
                       keep.f32(background_data, "background_data"), tw, th, int(bool(fast_math)),
                       _lib.FOVEATION[foveation], float(rings[0]), float(rings[1]))
    return keep, prims, st


def _request(device: torch.device, scene: int, eyes: list, images: list | None, tag: int, to_chw: bool) -> tuple:
    """The C request of one or two eyes; device tables of partial masks go to `device`."""
    if not 1 <= len(eyes) <= 2:
        raise ValueError("a request has one or two eyes")
    keep = _Keep(device)
    req = _lib.Request()
    req.scene = int(scene)
    req.n_eyes = len(eyes)
    req.tag = int(tag)
    shapes = []
    for i, v in enumerate(eyes):
        e = _eye_from(v, device, keep)
        h, w = int(v.height), int(v.width)
        shape = (3, h, w) if to_chw else (h, w, 3)
        if images is not None and images[i] is not None:
            img = images[i]
            if tuple(img.shape) != shape:
                raise ValueError(f"image {i} must have shape {shape}")
            e.image = keep.f32(img, f"image {i}")
        req.eyes[i] = e
        shapes.append(shape)
    if keep.refs:
        # device inputs made (or images last used) on PyTorch's stream: the frame waits for
        # this point of it, not for the whole device
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(device))
        keep.refs.append(ev)
        req.ready_event = ev.cuda_event
    return req, keep, shapes


def _completion(c: _lib.Completion, shapes: list, device: torch.device) -> Completion:
    imgs = []
    if c.status == 0:
        for i, shape in enumerate(shapes):
            ptr = c.images[i]
            imgs.append(torch.as_tensor(_DeviceArray(ptr, shape), device=device) if ptr else None)
    return Completion(int(c.ticket), int(c.tag), int(c.status), int(c.frame_views), float(c.submit_ms),
                      float(c.launch_ms), float(c.done_ms), c.message.decode(errors="replace"), imgs)


class Server:
    """Continuous-batching request server on one CUDA device (see the module docstring)."""

    def __init__(self, device: int | torch.device | None = None, hbm_budget_bytes: float = 150e9,
                 max_in_flight: int = 2, max_batch_requests: int = 8, blend_split: float = 0.0):
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        if dev.type != "cuda":
            raise ValueError("the server needs a CUDA device")
        self.device = torch.device("cuda", dev.index if dev.index is not None else torch.cuda.current_device())
        self._libh = _lib.load()
        cfg = _lib.ServerConfig(self.device.index, int(max_in_flight), int(max_batch_requests),
                                int(round(blend_split * 1000)), int(hbm_budget_bytes))
        out = _lib.vp()
        with torch.cuda.device(self.device):
            _lib.check(self._libh.fhtgs_server_create(C.byref(cfg), C.byref(out)))
        self.handle = out.value
        self._lock = threading.Lock()
        self._scenes: dict[int, tuple] = {}       # id -> (keep-alive, to_chw)
        self._pending: dict[int, tuple] = {}      # ticket -> (keep-alive, shapes)

    # ---- scenes ----
    def add_scene(self, positions, scales, rotations, opacities, sh_0, sh_rest, *, K: int = 8,
                  active_sh_bases: int = 16, near_plane: float = 0.2, far_plane: float = 100.0,
                  scale_modifier: float = 1.0, to_chw: bool = True, blur_periphery: bool = False,
                  aaa_mode: bool = False, fast_math: bool = True, background: BackgroundModel = BackgroundModel.NONE,
                  background_data: torch.Tensor | None = None, foveation: str = "reference",
                  rings: tuple[float, float] = (0.15, 0.4)) -> int:
        """Registers resident Gaussians (device tensors, fp32 or the fp16/bf16 storage).
        `foveation` / `rings`: as Renderer.set_foveation, for every request of the scene."""
        keep, prims, st = _scene_structs(self.device, positions, scales, rotations, opacities, sh_0, sh_rest, K=K,
                                         active_sh_bases=active_sh_bases, near_plane=near_plane,
                                         far_plane=far_plane, scale_modifier=scale_modifier, to_chw=to_chw,
                                         blur_periphery=blur_periphery, aaa_mode=aaa_mode, fast_math=fast_math,
                                         background=background, background_data=background_data,
                                         foveation=foveation, rings=rings)
        sid = C.c_int32(-1)
        _lib.check(self._libh.fhtgs_server_add_scene(self.handle, C.byref(prims), C.byref(st), C.byref(sid)))
        with self._lock:
            self._scenes[sid.value] = (keep, bool(to_chw))
        return sid.value

    def remove_scene(self, scene: int):
        _lib.check(self._libh.fhtgs_server_remove_scene(self.handle, int(scene)))

    # ---- requests ----
    def submit(self, scene: int, eyes: list, images: list | None = None, tag: int = 0) -> int:
        """Queues one request of 1 or 2 eyes; returns its ticket.  `images[i]` (optional) is a
        float32 device tensor the eye is rendered into; without it the server renders into an
        output buffer of its own, returned by `poll` and recycled by `release`."""
        return self.submit_prepared(self.prepare(scene, eyes, images, tag))

    def prepare(self, scene: int, eyes: list, images: list | None = None, tag: int = 0) -> tuple:
        """The C request of `submit` built ahead of time (for a caller that replays a trace)."""
        with self._lock:
            if scene not in self._scenes:
                raise _lib.FhtgsError(1, "unknown scene")
            to_chw = self._scenes[scene][1]
        return _request(self.device, scene, eyes, images, tag, to_chw)

    def submit_prepared(self, prepared: tuple) -> int:
        req, keep, shapes = prepared
        ticket = C.c_int64(0)
        _lib.check(self._libh.fhtgs_server_submit(self.handle, C.byref(req), C.byref(ticket)))
        with self._lock:
            self._pending[ticket.value] = (keep, shapes)
        return ticket.value

    def poll(self, max_completions: int = 64, wait_ms: int = 0) -> list[Completion]:
        """Finished requests (in completion order); waits up to wait_ms for the first."""
        buf = (_lib.Completion * max_completions)()
        n = C.c_int32(0)
        _lib.check(self._libh.fhtgs_server_poll(self.handle, buf, max_completions, int(wait_ms), C.byref(n)))
        out = []
        for k in range(n.value):
            c = buf[k]
            with self._lock:
                _, shapes = self._pending.pop(c.ticket, (None, []))
            out.append(_completion(c, shapes, self.device))
        return out

    def release(self, ticket: int):
        """Returns the server-owned outputs of a completed request to the pool (its image
        tensors must not be used afterwards)."""
        _lib.check(self._libh.fhtgs_server_release(self.handle, int(ticket)))

    def pause(self):
        """Queue requests without launching frames (running frames finish)."""
        _lib.check(self._libh.fhtgs_server_set_paused(self.handle, 1))

    def resume(self):
        _lib.check(self._libh.fhtgs_server_set_paused(self.handle, 0))

    def drain(self, timeout_ms: int = -1):
        _lib.check(self._libh.fhtgs_server_drain(self.handle, int(timeout_ms)))

    def stats(self) -> dict:
        s = _lib.ServerStats()
        _lib.check(self._libh.fhtgs_server_get_stats(self.handle, C.byref(s)))
        return {name: int(getattr(s, name)) for name, _ in _lib.ServerStats._fields_}

    def clock_ms(self) -> float:
        """The server's clock (ms since creation); completions are stamped with it."""
        return float(self._libh.fhtgs_server_clock_ms(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            self._libh.fhtgs_server_destroy(self.handle)
            self.handle = None
            self._pending.clear()
            self._scenes.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ServerGroup:
    """Replica group of request servers over several CUDA devices (fhtgs_server_group_*).

    Each device in `devices` runs one server (a device may be listed more than once: several
    replicas on one GPU).  `add_scene` keeps the caller's tensors on their device for the first
    replica there and copies them peer to peer into every other replica's HBM; `submit` routes a
    request, whole, to the replica with the least outstanding work (requests carrying device
    buffers stay on those buffers' device); `poll` returns completions of every replica with
    `replica` and `device` set.  Nothing crosses devices per frame."""

    def __init__(self, devices: list, hbm_budget_bytes: float = 150e9, max_in_flight: int = 2,
                 max_batch_requests: int = 8, blend_split: float = 0.0):
        self.devices = [torch.device("cuda", torch.device(d).index if not isinstance(d, int) else d) for d in devices]
        self._libh = _lib.load()
        ids = (C.c_int32 * len(self.devices))(*[d.index for d in self.devices])
        cfg = _lib.ServerConfig(0, int(max_in_flight), int(max_batch_requests), int(round(blend_split * 1000)),
                                int(hbm_budget_bytes))
        out = _lib.vp()
        _lib.check(self._libh.fhtgs_server_group_create(ids, len(self.devices), C.byref(cfg), C.byref(out)))
        self.handle = out.value
        self._lock = threading.Lock()
        self._scenes: dict[int, tuple] = {}    # id -> (keep-alive, to_chw, home device)
        self._pending: dict[int, tuple] = {}   # ticket -> (keep-alive, shapes)

    def __len__(self) -> int:
        return len(self.devices)

    def add_scene(self, positions, scales, rotations, opacities, sh_0, sh_rest, **settings) -> int:
        """As Server.add_scene; the tensors' device is the scene's home device."""
        home = positions.device
        defaults = dict(K=8, active_sh_bases=16, near_plane=0.2, far_plane=100.0, scale_modifier=1.0, to_chw=True,
                        blur_periphery=False, aaa_mode=False, fast_math=True, background=BackgroundModel.NONE,
                        background_data=None, foveation="reference", rings=(0.15, 0.4))
        unknown = set(settings) - set(defaults)
        if unknown:
            raise TypeError(f"unknown scene settings {sorted(unknown)}")
        defaults.update(settings)
        keep, prims, st = _scene_structs(home, positions, scales, rotations, opacities, sh_0, sh_rest, **defaults)
        sid = C.c_int32(-1)
        _lib.check(self._libh.fhtgs_server_group_add_scene(self.handle, home.index, C.byref(prims), C.byref(st),
                                                           C.byref(sid)))
        with self._lock:
            self._scenes[sid.value] = (keep, bool(defaults["to_chw"]), home)
        return sid.value

    def remove_scene(self, scene: int):
        _lib.check(self._libh.fhtgs_server_group_remove_scene(self.handle, int(scene)))

    def submit(self, scene: int, eyes: list, images: list | None = None, tag: int = 0) -> tuple[int, int]:
        """Queues one request; returns (ticket, replica).  Eyes with partial masks upload their
        tables to the scene's home device, which binds the request to replicas there."""
        with self._lock:
            if scene not in self._scenes:
                raise _lib.FhtgsError(1, "unknown scene")
            _, to_chw, home = self._scenes[scene]
        dev = images[0].device if images is not None and images[0] is not None else home
        req, keep, shapes = _request(dev, scene, eyes, images, tag, to_chw)
        ticket, replica = C.c_int64(0), C.c_int32(-1)
        _lib.check(self._libh.fhtgs_server_group_submit(self.handle, C.byref(req), C.byref(ticket), C.byref(replica)))
        with self._lock:
            self._pending[ticket.value] = (keep, shapes)
        return ticket.value, replica.value

    def poll(self, max_completions: int = 64, wait_ms: int = 0) -> list[Completion]:
        buf = (_lib.GroupCompletion * max_completions)()
        n = C.c_int32(0)
        _lib.check(self._libh.fhtgs_server_group_poll(self.handle, buf, max_completions, int(wait_ms), C.byref(n)))
        out = []
        for k in range(n.value):
            g = buf[k]
            with self._lock:
                _, shapes = self._pending.pop(g.completion.ticket, (None, []))
            c = _completion(g.completion, shapes, torch.device("cuda", g.device))
            c.replica, c.device = int(g.replica), int(g.device)
            out.append(c)
        return out

    def release(self, ticket: int):
        _lib.check(self._libh.fhtgs_server_group_release(self.handle, int(ticket)))

    def drain(self, timeout_ms: int = -1):
        _lib.check(self._libh.fhtgs_server_group_drain(self.handle, int(timeout_ms)))

    def stats(self, replica: int) -> dict:
        s = _lib.ServerStats()
        cost = C.c_int64(0)
        _lib.check(self._libh.fhtgs_server_group_get_stats(self.handle, int(replica), C.byref(s), C.byref(cost)))
        d = {name: int(getattr(s, name)) for name, _ in _lib.ServerStats._fields_}
        d["outstanding_cost"] = int(cost.value)
        return d

    def close(self):
        if getattr(self, "handle", None):
            self._libh.fhtgs_server_group_destroy(self.handle)
            self.handle = None
            self._pending.clear()
            self._scenes.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
