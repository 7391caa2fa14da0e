"""A stand-in frame server for testing the VapourSynth plugin (libsvpflow1_vs.so) without
VapourSynth: a VSAPI function table with entries at the byte offsets the reference plugin
reads (crates/svpflow1/src/vs.rs:48-65, analyse_filter.rs:194), maps, nodes, frames with
padded row pitches, and a driver that runs a filter's getFrame through the two activation
reasons (arInitial, then arAllFramesReady) the way a frame server does.

Handles for maps, nodes, frames and the core are opaque integers; the plugin only hands
them back to the table's functions. Frame planes are numpy buffers (stride x rows)."""
import ctypes as C

import numpy as np

VP = C.c_void_p
PF_GRAY8 = 1000010
AR_INITIAL, AR_ALL_FRAMES_READY = 0, 2

OFFSETS = {"free_frame": 48, "free_node": 56, "new_video_frame": 72, "create_filter": 136, "set_error": 144,
           "get_format_preset": 176, "get_frame_filter": 208, "request_frame_filter": 216, "get_stride": 240,
           "get_read_ptr": 248, "get_write_ptr": 256, "get_video_info": 304, "set_video_info": 312,
           "prop_get_int": 392, "prop_get_data": 408, "prop_get_data_size": 416, "prop_get_node": 424,
           "prop_set_int": 456}


class VideoInfo(C.Structure):  # vs.rs:76-86
    _fields_ = [("format", VP), ("fps_num", C.c_int64), ("fps_den", C.c_int64), ("width", C.c_int32),
                ("height", C.c_int32), ("num_frames", C.c_int32), ("flags", C.c_int32)]


CREATE = C.CFUNCTYPE(C.c_ssize_t, VP, VP, VP, VP, VP)
CONFIG = C.CFUNCTYPE(None, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int32, C.c_int32, VP)
REGISTER = C.CFUNCTYPE(None, C.c_char_p, C.c_char_p, VP, VP, VP)
INIT = C.CFUNCTYPE(None, VP, VP, C.POINTER(VP), VP, VP, VP)
GETFRAME = C.CFUNCTYPE(VP, C.c_int32, C.c_int32, C.POINTER(VP), C.POINTER(VP), VP, VP, VP)
FREE = C.CFUNCTYPE(None, VP, VP, VP)
T = {
    "create_filter": C.CFUNCTYPE(None, VP, VP, C.c_char_p, VP, VP, VP, C.c_int32, C.c_int32, VP, VP),
    "set_error": C.CFUNCTYPE(None, VP, C.c_char_p),
    "get_video_info": C.CFUNCTYPE(VP, VP),
    "set_video_info": C.CFUNCTYPE(None, VP, C.c_int32, VP),
    "prop_get_int": C.CFUNCTYPE(C.c_int64, VP, C.c_char_p, C.c_int32, C.POINTER(C.c_int32)),
    "prop_get_data": C.CFUNCTYPE(VP, VP, C.c_char_p, C.c_int32, C.POINTER(C.c_int32)),
    "prop_get_data_size": C.CFUNCTYPE(C.c_int32, VP, C.c_char_p, C.c_int32, C.POINTER(C.c_int32)),
    "prop_get_node": C.CFUNCTYPE(VP, VP, C.c_char_p, C.c_int32, C.POINTER(C.c_int32)),
    "prop_set_int": C.CFUNCTYPE(C.c_int32, VP, C.c_char_p, C.c_int64, C.c_int32),
    "free_frame": C.CFUNCTYPE(None, VP),
    "free_node": C.CFUNCTYPE(None, VP),
    "get_frame_filter": C.CFUNCTYPE(VP, C.c_int32, VP, VP),
    "new_video_frame": C.CFUNCTYPE(VP, VP, C.c_int32, C.c_int32, VP, VP),
    "get_stride": C.CFUNCTYPE(C.c_int32, VP, C.c_int32),
    "get_read_ptr": C.CFUNCTYPE(VP, VP, C.c_int32),
    "get_write_ptr": C.CFUNCTYPE(VP, VP, C.c_int32),
    "request_frame_filter": C.CFUNCTYPE(None, C.c_int32, VP, VP),
    "get_format_preset": C.CFUNCTYPE(VP, C.c_int32, VP),
}


class NodeRef(int):
    """A node handle passed as a filter argument."""


class Frame:
    def __init__(self, fmt, width, height, align, fill=0xCD):
        self.fmt, self.width, self.height = fmt, width, height
        cw, ch = width // 2, height // 2
        dims = [(width, height)] if fmt == "gray8" else [(width, height), (cw, ch), (cw, ch)]
        self.strides, self.planes = [], []
        for w, h in dims:
            st = max(((w + align - 1) // align) * align, align)
            self.strides.append(st)
            self.planes.append(np.full(st * max(h, 1), fill, dtype=np.uint8))
        self.rows = [h for _, h in dims]

    def plane(self, p):
        """The plane as a (rows, stride) array including the row padding."""
        return self.planes[p][: self.strides[p] * self.rows[p]].reshape(self.rows[p], self.strides[p])


class Node:
    def __init__(self, vi):
        self.vi = vi


class SourceNode(Node):
    def __init__(self, vi, frames):
        super().__init__(vi)
        self.frames = frames  # frame handles


class FilterNode(Node):
    def __init__(self, name, getframe, free, instance, mode):
        super().__init__(VideoInfo())
        self.name, self.getframe, self.free, self.mode = name, getframe, free, mode
        self.instance = VP(instance)
        self.frame_data = VP(0)


class Server:
    """The fake frame server: its VSAPI table, objects and a frame driver."""

    def __init__(self, align=64):
        self.align = align
        self.objs = {}
        self._next = 0x10000
        self.errors = []
        self.freed_frames = 0
        self.freed_nodes = 0
        self.core = self._new(object())
        self.fmt_yuv = C.create_string_buffer(b"YUV420P8")
        self.fmt_gray = C.create_string_buffer(b"Gray8")
        self.formats = {C.addressof(self.fmt_yuv): "yuv420p8", C.addressof(self.fmt_gray): "gray8"}
        self.gray_preset = True
        self._keep = []
        self.table = (VP * 64)()
        self._cbs = {}
        for name, off in OFFSETS.items():
            cb = T[name](getattr(self, "_" + name))
            self._cbs[name] = cb
            self.table[off // 8] = C.cast(cb, VP).value

    @property
    def vsapi(self):
        return C.addressof(self.table)

    def _new(self, obj) -> int:
        self._next += 16
        self.objs[self._next] = obj
        return self._next

    # ---- maps
    def new_map(self, props=None) -> int:
        m = {}
        for k, v in (props or {}).items():
            if isinstance(v, (bytes, str)):
                b = v.encode() if isinstance(v, str) else v
                buf = C.create_string_buffer(b, len(b))
                self._keep.append(buf)
                m[k] = ("data", buf, len(b))
            elif isinstance(v, NodeRef):
                m[k] = ("node", int(v))
            else:
                m[k] = ("int", int(v))
        return self._new(m)

    def map(self, h) -> dict:
        return self.objs[h]

    # ---- clips
    def source_clip(self, frames_i420: np.ndarray, width: int, height: int, fps=(30000, 1001)) -> int:
        """A YUV420P8 clip node from packed I420 frames (rows laid out at padded pitches)."""
        handles = []
        cw, ch = width // 2, height // 2
        for f in frames_i420:
            fr = Frame("yuv420p8", width, height, self.align, fill=0)
            fr.plane(0)[:, :width] = f[: width * height].reshape(height, width)
            fr.plane(1)[:, :cw] = f[width * height: width * height + cw * ch].reshape(ch, cw)
            fr.plane(2)[:, :cw] = f[width * height + cw * ch:].reshape(ch, cw)
            handles.append(self._new(fr))
        vi = VideoInfo(C.addressof(self.fmt_yuv), fps[0], fps[1], width, height, len(handles), 0)
        return NodeRef(self._new(SourceNode(vi, handles)))

    def frame(self, h) -> Frame:
        return self.objs[h]

    # ---- driving a filter
    def get_frame(self, node_h: int, n: int) -> int:
        node = self.objs[node_h]
        n = min(max(n, 0), node.vi.num_frames - 1)  # requests past the end get the last frame
        if isinstance(node, SourceNode):
            return node.frames[n]
        ctx = {"requests": []}
        ctx_h = self._new(ctx)
        r = node.getframe(n, AR_INITIAL, C.byref(node.instance), C.byref(node.frame_data), ctx_h, self.core,
                          self.vsapi)
        assert not r
        ctx["ready"] = {(nh, k): self.get_frame(nh, k) for (k, nh) in ctx["requests"]}
        out = node.getframe(n, AR_ALL_FRAMES_READY, C.byref(node.instance), C.byref(node.frame_data), ctx_h,
                            self.core, self.vsapi)
        return out or 0

    def free_filter(self, node_h: int):
        node = self.objs[node_h]
        node.free(node.instance, self.core, self.vsapi)

    # ---- VSAPI entries
    def _set_error(self, m, msg):
        self.errors.append(msg.decode())
        self.objs[m]["_error"] = msg.decode()

    def _get_video_info(self, node_h):
        return C.addressof(self.objs[node_h].vi)

    def _set_video_info(self, vi_p, n, node_h):
        vi = C.cast(vi_p, C.POINTER(VideoInfo)).contents
        C.memmove(C.addressof(self.objs[node_h].vi), C.addressof(vi), C.sizeof(VideoInfo))

    def _lookup(self, m, key, idx, err, kind):
        v = self.objs[m].get(key.decode())
        if v is None or v[0] != kind or idx != 0:
            if err:
                err[0] = 1
            return None
        if err:
            err[0] = 0
        return v

    def _prop_get_int(self, m, key, idx, err):
        v = self._lookup(m, key, idx, err, "int")
        return v[1] if v else 0

    def _prop_get_data(self, m, key, idx, err):
        v = self._lookup(m, key, idx, err, "data")
        return C.addressof(v[1]) if v else None

    def _prop_get_data_size(self, m, key, idx, err):
        v = self._lookup(m, key, idx, err, "data")
        return v[2] if v else -1

    def _prop_get_node(self, m, key, idx, err):
        v = self._lookup(m, key, idx, err, "node")
        return v[1] if v else None

    def _prop_set_int(self, m, key, value, append):
        self.objs[m][key.decode()] = ("int", value)
        return 0

    def _create_filter(self, in_m, out_m, name, init, getframe, free, mode, flags, instance, core):
        node = FilterNode(name.decode(), GETFRAME(getframe), FREE(free), instance, mode)
        h = self._new(node)
        INIT(init)(in_m, out_m, C.byref(node.instance), h, core, self.vsapi)
        self.objs[out_m]["clip"] = ("node", NodeRef(h))

    def _free_frame(self, f):
        self.freed_frames += 1

    def _free_node(self, n):
        self.freed_nodes += 1

    def _request_frame_filter(self, n, node_h, ctx_h):
        n = min(max(n, 0), self.objs[node_h].vi.num_frames - 1)
        self.objs[ctx_h]["requests"].append((n, node_h))

    def _get_frame_filter(self, n, node_h, ctx_h):
        ready = self.objs[ctx_h]["ready"]
        node = self.objs[node_h]
        n = min(max(n, 0), node.vi.num_frames - 1)
        return ready.get((node_h, n)) or self.get_frame(node_h, n)

    def _new_video_frame(self, fmt, w, h, propsrc, core):
        return self._new(Frame(self.formats.get(fmt, "yuv420p8"), w, h, self.align))

    def _get_stride(self, f, p):
        return self.objs[f].strides[p]

    def _get_read_ptr(self, f, p):
        return self.objs[f].planes[p].ctypes.data

    def _get_write_ptr(self, f, p):
        return self.objs[f].planes[p].ctypes.data

    def _get_format_preset(self, fid, core):
        return C.addressof(self.fmt_gray) if (fid == PF_GRAY8 and self.gray_preset) else None


class Plugin:
    """libsvpflow1_vs.so loaded and registered against a Server."""

    def __init__(self, path: str, server: Server):
        self.lib = C.CDLL(path)
        self.srv = server
        self.config_calls, self.functions = [], {}
        self.lib.svpGetVersion.restype = C.c_int64
        self.lib.VapourSynthPluginInit.argtypes = [VP, VP, VP]

        def config(ident, ns, name, api, ro, plugin):
            self.config_calls.append((ident.decode(), ns.decode(), name.decode(), api, ro, plugin))

        def register(name, args, create, user, plugin):
            self.functions[name.decode()] = (args.decode(), CREATE(create))

        self._cfg, self._reg = CONFIG(config), REGISTER(register)
        self.lib.VapourSynthPluginInit(C.cast(self._cfg, VP), C.cast(self._reg, VP), 0x1234)

    def invoke(self, name: str, args: dict):
        """Calls the filter's create function; returns (out map dict, out map handle)."""
        in_m = self.srv.new_map(args)
        out_m = self.srv.new_map()
        self.functions[name][1](in_m, out_m, None, self.srv.core, self.srv.vsapi)
        return self.srv.map(out_m), out_m
