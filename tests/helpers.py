"""Shared helpers of the test suite."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def unpack_mask(packed, shape):
    n = int(np.prod(shape))
    return np.unpackbits(packed)[:n].reshape(tuple(int(s) for s in shape)).astype(np.uint8)


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    z = np.load(path, allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["mask"] = unpack_mask(d["mask"], d["shape"])
    return d


def spheres(shape, phi, r, seed):
    from lbm_b200 import geometry as G

    return G.overlapping_spheres(shape, phi, r, seed)


def _open_by_any_process(path):
    """Whether some process holds `path` open (a scan of /proc/*/fd)."""
    real = os.path.realpath(path)
    for pid in os.listdir("/proc"):
        if not pid.isdigit():
            continue
        try:
            fds = os.listdir(f"/proc/{pid}/fd")
        except OSError:
            continue
        for fd in fds:
            try:
                if os.readlink(f"/proc/{pid}/fd/{fd}") == real:
                    return True
            except OSError:
                pass
    return False


class InputVersions:
    """A named pipe at `path` whose k-th opening reads texts[k] (the last text
    for any later opening): a program that reads its INPUT file again while
    it runs (the colour-gradient program's input_dynamic) sees the versions
    in the order it opens the file, at the steps it opens it.  Each version
    is written whole and closed (the reader sees its end), and the next
    opening is served only after every reader of the previous one closed.
    `served` counts the openings served."""

    def __init__(self, path, texts):
        import threading

        self.path, self.texts, self.served = path, [t.encode() for t in texts], 0
        self._stop = threading.Event()
        os.mkfifo(path)
        self._thread = threading.Thread(target=self._feed, daemon=True)
        self._thread.start()

    def _feed(self):
        import time

        while True:
            fd = os.open(self.path, os.O_WRONLY)  # waits for a reader
            if self._stop.is_set():
                os.close(fd)
                return
            data = self.texts[min(self.served, len(self.texts) - 1)]
            try:
                while data:
                    data = data[os.write(fd, data):]
            except BrokenPipeError:
                pass
            os.close(fd)
            self.served += 1
            while _open_by_any_process(self.path) and not self._stop.is_set():
                time.sleep(0.001)

    def close(self):
        self._stop.set()
        # a reader of our own lets a writer waiting in open() go on and stop
        fd = os.open(self.path, os.O_RDONLY | os.O_NONBLOCK)
        self._thread.join(timeout=10)
        os.close(fd)
        os.unlink(self.path)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
