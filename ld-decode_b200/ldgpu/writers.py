"""The reference's per-field output files, for the batched path.

LDdecode opens them in its constructor (lddecode/core.py:3577-3590) and
appends one field at a time in writeout (core.py:3918-4015):

  <name>.tbc    the uint16 TBC picture of every field, as produced
                (outfile_video.write(picture), core.py:4002);
  <name>.pcm    the interleaved int16 analog audio of every field
                (core.py:4014-4015);
  <name>.prefm  the int16 EFM samples of every field before the EFM PLL
                (write_pre_efm, core.py:3585-3586, 3921-3922);
  RF TBC        int16 lines (Field.rf_tbc); the reference pipes them to
                ffmpeg for a .tbc.ldf (core.py:3587-3589, 4005-4012), here
                they go to <name>.rftbc as the raw samples ffmpeg would get.

  <name>.efm    the EFM PLL's T-values of every field's EFM samples
                (efm_pll.EFM_PLL over the fields in order, core.py:3583,
                3924-3925), from the native PLL (ldgpu.efm.EFM_PLL).

The .tbc.db metadata is SQLite and stays with the reference's own code.
The batched path hands whole batches of fields over at once;
`FieldWriter(..., background=True)` writes them on a host thread so that
the files are written while the GPU works on the next batch.
"""

import queue
import threading

import numpy as np


class FieldWriter:
    """Appends fields to the reference's output files (see the module
    docstring).  `audio`, `efm`, `prefm`, `rftbc` select the optional
    files, as the reference's analog_audio, digital_audio, write_pre_efm
    and write_rf_tbc do."""

    def __init__(self, fname_out, audio=False, prefm=False, rftbc=False, background=False, efm=False):
        self.fname_out = fname_out
        self.video = open(fname_out + ".tbc", "wb")
        self.audio = open(fname_out + ".pcm", "wb") if audio else None
        self.prefm = open(fname_out + ".prefm", "wb") if prefm else None
        self.rftbc = open(fname_out + ".rftbc", "wb") if rftbc else None
        self.efm = open(fname_out + ".efm", "wb") if efm else None
        self.efm_pll = None
        if efm:
            from .efm import EFM_PLL
            self.efm_pll = EFM_PLL()
        self.fields_written = 0
        self._q = None
        self._thread = None
        self._error = None
        if background:
            self._q = queue.Queue(maxsize=4)
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()

    # ---- writing

    @staticmethod
    def _check(a, dtype, what):
        a = np.asarray(a)
        if a.dtype != dtype:
            raise TypeError(f"{what} must be {np.dtype(dtype).name}, got {a.dtype}")
        return np.ascontiguousarray(a)

    def _write_field(self, picture, audio, efm, rftbc):
        self.video.write(self._check(picture, np.uint16, "picture").tobytes())
        if audio is not None and self.audio is not None:
            self.audio.write(self._check(audio, np.int16, "audio").tobytes())
        if efm is not None and self.prefm is not None:
            self.prefm.write(self._check(efm, np.int16, "efm").tobytes())
        if efm is not None and self.efm is not None:
            self.efm.write(self.efm_pll.process(self._check(efm, np.int16, "efm")).tobytes())
        if rftbc is not None and self.rftbc is not None:
            self.rftbc.write(self._check(rftbc, np.int16, "rftbc").tobytes())
        self.fields_written += 1

    def _write_batch(self, pictures, audio, efm, rftbc):
        n = len(pictures)
        for i in range(n):
            self._write_field(pictures[i], None if audio is None else audio[i], None if efm is None else efm[i],
                              None if rftbc is None else rftbc[i])

    def write(self, picture, audio=None, efm=None, rftbc=None):
        """One field, in order (LDdecode.writeout)."""
        self.write_batch([picture], None if audio is None else [audio], None if efm is None else [efm],
                         None if rftbc is None else [rftbc])

    def write_batch(self, pictures, audio=None, efm=None, rftbc=None):
        """Fields in order: `pictures` a (n, lines * width) uint16 array or a
        list of pictures; `audio`, `efm`, `rftbc` lists of per-field arrays
        (or None).  With background=True the arrays must not be modified
        until flush() (they are written later, from a host thread)."""
        self._raise()
        if self._q is None:
            self._write_batch(pictures, audio, efm, rftbc)
        else:
            self._q.put((pictures, audio, efm, rftbc))

    # ---- background thread

    def _run(self):
        while True:
            item = self._q.get()
            try:
                if item is None:
                    return
                if self._error is None:
                    self._write_batch(*item)
            except Exception as e:  # reported by the next call on the caller's thread
                self._error = e
            finally:
                self._q.task_done()

    def _raise(self):
        if self._error is not None:
            e, self._error = self._error, None
            raise e

    def flush(self):
        """Wait until every batch handed over so far is in the files."""
        if self._q is not None:
            self._q.join()
        self._raise()
        for f in (self.video, self.audio, self.prefm, self.rftbc, self.efm):
            if f is not None:
                f.flush()

    def close(self):
        try:
            self.flush()
        finally:
            if self._thread is not None:
                self._q.put(None)
                self._thread.join()
                self._thread = None
            for f in (self.video, self.audio, self.prefm, self.rftbc, self.efm):
                if f is not None:
                    f.close()
            if self.efm_pll is not None:
                self.efm_pll.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
