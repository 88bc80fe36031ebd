"""Stand-ins for cuacd_b200.Context in the command-line tests (no GPU).

Each factory is a module-level function, so the pipeline's spawned
decomposer can unpickle it.  Failures are made on the host: a Python
exception, or the process killing itself with SIGKILL (which is what a
native crash looks like to the supervisor)."""
import os
import signal

import numpy as np

BOX_T = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [2, 3, 7], [2, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.int32)


def box_of(v):
    lo, hi = v.min(0), v.max(0)
    return np.array([[lo[0], lo[1], lo[2]], [hi[0], lo[1], lo[2]], [hi[0], hi[1], lo[2]], [lo[0], hi[1], lo[2]],
                     [lo[0], lo[1], hi[2]], [hi[0], lo[1], hi[2]], [hi[0], hi[1], hi[2]], [lo[0], hi[1], hi[2]]],
                    np.float32)


class FakeContext:
    """Every mesh gives two parts: (the mesh, its hull = the mesh) and
    (its bounding box, the box).  fail=True raises on every call; a mesh of
    exactly `crash_nv` vertices kills the process.  The audit flags a mesh
    with an odd triangle count; the remesh replaces a mesh by its bounding
    box."""

    def __init__(self, fail=False, crash_nv=-1):
        self.fail, self.crash_nv, self.closed = fail, crash_nv, False

    def check_mesh(self, v, t):
        odd = len(t) % 2 == 1
        return {"needs_remesh": odd, "flags": 4 if odd else 0}

    def preprocess(self, v, t, resolution=64):
        assert resolution & (resolution - 1) == 0
        return box_of(v), BOX_T

    def lookahead_decompose(self, v, t, **kw):
        if len(v) == self.crash_nv:
            os.kill(os.getpid(), signal.SIGKILL)
        if self.fail:
            raise RuntimeError("injected failure")
        b = box_of(v)
        return [(v, t, v, t), (b, BOX_T, b, BOX_T)]

    def pool_usage(self):
        return 3 << 20

    def close(self):
        self.closed = True


def ok_factory(device, pool_bytes):
    return FakeContext()


def crash_factory(device, pool_bytes):
    return FakeContext(crash_nv=5)


_opened = [0]


def flaky_factory(device, pool_bytes):
    """The first context of a process fails every call; later ones work."""
    _opened[0] += 1
    return FakeContext(fail=_opened[0] == 1)


def failing_factory(device, pool_bytes):
    return FakeContext(fail=True)


# ---- supervisor tests ------------------------------------------------------
class FakeProc:
    """Process stand-in: alive for `ticks` liveness polls, then exited with
    `code`."""

    def __init__(self, code, ticks=0):
        self.code, self.ticks, self.exitcode, self.terminated = code, ticks, None, False

    def is_alive(self):
        if self.ticks > 0:
            self.ticks -= 1
            return True
        self.exitcode = self.code
        return False

    def terminate(self):
        self.terminated = True
        self.ticks = 0

    def join(self, timeout=None):
        pass


def exit_after_one_item(q):
    q.get()
    os._exit(3)                        # no traceback, no end-of-stream marker


def wait_for_item(q):
    q.get()
