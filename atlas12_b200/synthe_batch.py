"""SYNTHE spectra of many atmospheres, each with its own window and line list.

The reference synthesises one spectrum per process (scripts/synthe.sh:35).
Here `lanes` library contexts, each with its own CUDA stream and its own
device buffers, are driven by one host thread each (the ctypes calls release
the interpreter lock), so the binning, continuum, line-opacity and spectrum
launches of different atmospheres overlap on the GPU: a small window no
longer leaves most of the SMs idle while its host-side steps run.  Every
spectrum is computed exactly as by synthe.Synthe.run on its own.

    sb = SyntheBatch(device=0, operators=tables, lanes=8)
    spectra = sb.run(cases)          # list of (wave_A, flux, cont_flux)
"""
import queue
import threading

from . import _lib
from . import synthe as S


class SyntheBatch:
    def __init__(self, device, operators, lanes=8, precision=_lib.PREC_MIXED, hydrogen_tables=None, stehle=None):
        """hydrogen_tables (the s_* arrays) and stehle (read_stehle_dir's list)
        go to every lane, for cases that carry unit-19 hydrogen records."""
        self.lanes = [S.Synthe(_lib.Context(device, precision), operators) for _ in range(max(1, int(lanes)))]
        if hydrogen_tables is not None:
            for syn in self.lanes:
                syn.set_hydrogen_tables(hydrogen_tables, stehle)

    def run(self, cases, keep_opacity=False):
        """Spectra of every case (synthetic.synthe_case dicts), in order."""
        out = [None] * len(cases)
        todo = queue.Queue()
        for i in range(len(cases)):
            todo.put(i)
        errors = []

        def work(syn):
            while True:
                try:
                    i = todo.get_nowait()
                except queue.Empty:
                    return
                try:
                    wave, flux, cflux, op = syn.run(cases[i])
                    out[i] = (wave, flux, cflux, op) if keep_opacity else (wave, flux, cflux)
                except Exception as e:  # reported after every lane has stopped
                    errors.append((i, e))

        threads = [threading.Thread(target=work, args=(syn,)) for syn in self.lanes]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            i, e = errors[0]
            raise RuntimeError(f"atmosphere {i}: {e}") from e
        return out

    def close(self):
        for syn in self.lanes:
            syn.ctx.close()
        self.lanes = []
