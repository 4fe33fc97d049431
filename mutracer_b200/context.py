"""Python mirror of the persistent context API (native/include/mutracer-context.h):
commit a flattened buffer bundle, render or submit/poll jobs, read pixels."""
import ctypes as C

import numpy as np

from . import abi

_ERR = 512


def _err():
    return C.create_string_buffer(_ERR)


def default_settings():
    s = abi.RenderSettings()
    abi.check(abi.lib().mt_render_settings_default(C.byref(s)))
    return s


class Context:
    def __init__(self):
        e = _err()
        h = C.c_uint64()
        abi.check(abi.lib().mt_context_create(C.byref(h), e, _ERR), e)
        self.handle = h.value

    def commit(self, host_scene, settings=None):
        e = _err()
        abi.check(abi.lib().mt_context_commit_bundle(self.handle, C.byref(host_scene.bundle),
                                                     C.byref(settings) if settings is not None else None, e, _ERR), e)

    def commit_descriptor(self, data, settings=None):
        """mt_context_commit / mt_context_commit_with_settings on a scene
        descriptor v8 (bytes, e.g. mutracer_b200.descriptor.Descriptor)."""
        e = _err()
        buf = np.frombuffer(bytes(data), np.uint8)
        ptr = C.c_void_p(buf.ctypes.data) if buf.size else None
        if settings is None:
            abi.check(abi.lib().mt_context_commit(self.handle, ptr, buf.size, e, _ERR), e)
        else:
            abi.check(abi.lib().mt_context_commit_with_settings(self.handle, ptr, buf.size, C.byref(settings), e,
                                                                _ERR), e)

    def render(self, samples):
        e = _err()
        abi.check(abi.lib().mt_context_render(self.handle, samples, e, _ERR), e)

    def reset(self):
        e = _err()
        abi.check(abi.lib().mt_context_reset(self.handle, e, _ERR), e)

    def wait(self, timeout_ms=0xFFFFFFFF):
        e = _err()
        abi.check(abi.lib().mt_context_wait(self.handle, timeout_ms, e, _ERR), e)

    def info(self):
        s = abi.ContextSnapshot()
        s.struct_size = C.sizeof(abi.ContextSnapshot)
        e = _err()
        abi.check(abi.lib().mt_context_info(self.handle, C.byref(s), e, _ERR), e)
        return s

    def read_pixels(self, kind=abi.MT_IMAGE_HDR, out=None):
        e = _err()
        need = C.c_size_t()
        abi.check(abi.lib().mt_context_read_pixels(self.handle, kind, None, 0, C.byref(need), e, _ERR), e)
        info = self.info()
        if out is None:
            out = np.empty((info.height, info.width, 4), dtype=np.float32)
        abi.check(abi.lib().mt_context_read_pixels(self.handle, kind, out.ctypes.data, out.nbytes, C.byref(need),
                                                   e, _ERR), e)
        return out

    def submit(self, samples):
        e = _err()
        j = C.c_uint64()
        abi.check(abi.lib().mt_context_submit(self.handle, samples, C.byref(j), e, _ERR), e)
        return Job(j.value)

    def destroy(self):
        if self.handle:
            e = _err()
            abi.check(abi.lib().mt_context_destroy(self.handle, e, _ERR), e)
            self.handle = 0


class Job:
    def __init__(self, handle):
        self.handle = handle

    def poll(self, max_new_samples=64):
        e = _err()
        abi.check(abi.lib().mt_job_poll(self.handle, max_new_samples, e, _ERR), e)

    def info(self):
        s = abi.JobSnapshot()
        s.struct_size = C.sizeof(abi.JobSnapshot)
        e = _err()
        abi.check(abi.lib().mt_job_info(self.handle, C.byref(s), e, _ERR), e)
        return s

    def cancel(self):
        e = _err()
        abi.check(abi.lib().mt_job_cancel(self.handle, e, _ERR), e)
