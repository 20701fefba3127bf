"""Bank search: a whole orbital bank over one or more series (possibly of
different lengths) in one captured CUDA graph -- the batched form of the
reference's bank loop (src/workunit_main.cpp:77-93)."""
import ctypes

import numpy as np

from ._lib import CANDIDATE, BrpError, Params, as_params, check, lib, ptr


class Bank:
    def __init__(self, lengths, unpadded, max_templates, capacity=4096, device=-1):
        L = lib()
        self._b = None
        self.n = np.ascontiguousarray(lengths, dtype=np.uint32)
        self.unpadded = np.ascontiguousarray(unpadded, dtype=np.uint32)
        self.max_templates = int(max_templates)
        self.capacity = int(capacity)
        b = ctypes.c_void_p()
        st = L.brp_cuda_bank_create(self.n.size, ptr(self.n), ptr(self.unpadded), max_templates, capacity, device,
                                    ctypes.byref(b))
        check(st, lambda: L.brp_cuda_bank_last_error(None).decode())
        self._b = b
        self._out = np.empty(0, CANDIDATE)

    def _err(self):
        return lib().brp_cuda_bank_last_error(self._b).decode()

    def close(self):
        if self._b:
            lib().brp_cuda_bank_destroy(self._b)
            self._b = None

    def __del__(self):
        self.close()

    def set_series(self, index, series):
        x = np.ascontiguousarray(series, dtype=np.float32)
        if x.size != self.unpadded[index]:
            raise BrpError(4, "series length mismatch")
        check(lib().brp_cuda_bank_set_series(self._b, index, ptr(x)), self._err)

    @staticmethod
    def params_array(templates):
        """A ctypes array of the templates (reusable across runs)."""
        return (Params * len(templates))(*[as_params(t) for t in templates])

    def run(self, templates, series_of=None, out=None):
        """Searches every template; returns (candidates per template, counts, status).
        Raises BrpError when a template overflowed or resampled out of range."""
        flat, offs, counts, status = self.run_flat(templates, series_of, out)
        return [flat[offs[t]:offs[t + 1]] for t in range(len(counts))], counts, status

    def run_flat(self, templates, series_of=None, out=None):
        """As run(), returning the candidates back to back: (candidates,
        offsets[count + 1], counts, status).  `templates` may be a list of
        Params or an array from params_array()."""
        self.submit(templates, series_of)
        return self.wait(out)

    def submit(self, templates, series_of=None):
        """Enqueues a run of the bank and returns at once (brp_cuda_bank_submit);
        wait() collects it.  set_series() meanwhile uploads into the buffer the
        run does not read, for the next submit."""
        arr = templates if isinstance(templates, ctypes.Array) else self.params_array(templates)
        count = len(arr)
        so = np.zeros(count, np.uint32) if series_of is None else np.ascontiguousarray(series_of, dtype=np.uint32)
        check(lib().brp_cuda_bank_submit(self._b, arr, ptr(so), count), self._err)
        self._submitted = count

    def wait(self, out=None):
        """Blocks until the submitted run is done: (candidates, offsets[count + 1],
        counts, status) as run_flat()."""
        count = getattr(self, "_submitted", 0)
        if not count:
            raise BrpError(4, "no submitted run to wait for")
        self._submitted = 0
        counts = np.zeros(count, np.uint32)
        status = np.zeros(count, np.uint32)
        cap = count * self.capacity
        if out is None:
            out = np.empty(cap, CANDIDATE)
        st = lib().brp_cuda_bank_wait(self._b, ptr(out), out.size, ptr(counts), ptr(status))
        if st and st != 2:
            check(st, self._err)
        offs = np.zeros(count + 1, np.int64)
        offs[1:] = np.cumsum(np.minimum(counts, self.capacity).astype(np.int64))
        flat = out[:offs[-1]]
        if st:
            e = BrpError(st, self._err())
            e.counts, e.status = counts, status
            e.candidates = [flat[offs[t]:offs[t + 1]] for t in range(count)]
            raise e
        return flat, offs, counts, status

    def configure(self, n, pass1=0, pass2=0, group=0, chains=0):
        """Selects compiled pass configurations, templates per launch and
        parallel launch chains for length n."""
        check(lib().brp_cuda_bank_configure(self._b, n, pass1, pass2, group, chains), self._err)

    def set_toplist_filter(self, rows=100):
        """Return only the candidates that can reach a per-series toplist of
        `rows` rows per level (0: all candidates); counts become the kept counts."""
        check(lib().brp_cuda_bank_set_toplist_filter(self._b, rows), self._err)

    def set_wait_limits(self, device_polls=1 << 22, host_seconds=300.0):
        """Bounds of the run's waits: the host deadline of run()/profile() and
        the poll bound of a kernel's first wait for its own asynchronous work
        (0 gives up at once; the template's status then has STATUS_WAIT_TIMEOUT)."""
        check(lib().brp_cuda_bank_set_wait_limits(self._b, device_polls, host_seconds), self._err)

    def launch(self):
        """Replays the last run's graph on the device only (no copies, no wait)."""
        check(lib().brp_cuda_bank_launch(self._b), self._err)

    def profile(self):
        """Per-kernel device time of one eager replay of the last run:
        ({"pass1", "pass2", "harmonic", "compact"} -> ms, launches per kind)."""
        ms = np.zeros(4, np.float64)
        launches = np.zeros(4, np.uint32)
        check(lib().brp_cuda_bank_profile(self._b, ptr(ms), ptr(launches)), self._err)
        names = ("pass1", "pass2", "harmonic", "compact")
        return dict(zip(names, ms.tolist())), dict(zip(names, launches.tolist()))

    @property
    def stream(self):
        return lib().brp_cuda_bank_stream(self._b)

    @property
    def kernels_per_run(self):
        return int(lib().brp_cuda_bank_kernels_per_run(self._b))
