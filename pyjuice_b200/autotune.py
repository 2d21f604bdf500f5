"""Launch-shape autotuner: the first time a kernel runs with a given shape key, every
candidate launch shape is timed on the device and the fastest is kept for that key.

Keys describe the work, not the layer: kernel family, mode, precision form, number of
tiles, tallest tile, batch size (``SumLayer`` builds them). Candidates produce the same
results (they only change how samples and tiles map to CTAs); accumulating launches are
tuned on scratch buffers (the caller's ``run`` decides where a candidate writes). Timing
uses CUDA events on the current stream: two warm-up runs per candidate, then the median of
``reps`` timed runs. Nothing is tuned while a CUDA graph is being captured: a key not yet
tuned then takes the first candidate (the static default) and is tuned at its next eager
launch. ``PCB_AUTOTUNE=0`` switches tuning off (static defaults); ``PCB_AUTOTUNE_CACHE``
names a JSON file the choices are read from and written to, so that later processes skip
the timing.

The reference tunes nothing at run time: its tile sizes are fixed expressions of the layer
shape (src/pyjuice/layer/sum_layer.py:831-840, 1912-1921).
"""

from __future__ import annotations

import json
import os
import statistics
from typing import Callable, Hashable, Sequence

import torch


class Autotuner:
    def __init__(self):
        self.enabled = os.environ.get("PCB_AUTOTUNE", "1") != "0"
        self.reps = 5
        self.choices = {}
        self.timings = {}
        self._path = os.environ.get("PCB_AUTOTUNE_CACHE")
        if self._path and os.path.exists(self._path):
            with open(self._path) as f:
                for k, v in json.load(f).items():
                    self.choices[k] = tuple(v) if isinstance(v, list) else v

    @staticmethod
    def _key(key: Sequence[Hashable]) -> str:
        return "|".join(str(k) for k in key)

    def pick(self, key: Sequence[Hashable], candidates: Sequence, run: Callable[[object], None]):
        """The chosen candidate for ``key`` (timing ``run(candidate)`` for each candidate on the
        first eager call). ``run`` must launch on the current stream and leave its outputs
        equal for every candidate, or write them to scratch."""
        k = self._key(key)
        if k in self.choices:
            return self.choices[k]
        if not self.enabled or len(candidates) == 1:
            return candidates[0]
        if torch.cuda.is_current_stream_capturing():
            return candidates[0]
        times = []
        for cand in candidates:
            try:
                for _ in range(2):
                    run(cand)
                ts = []
                for _ in range(self.reps):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    run(cand)
                    e1.record()
                    e1.synchronize()
                    ts.append(e0.elapsed_time(e1))
                times.append(statistics.median(ts))
            except RuntimeError:  # a candidate the library rejects for this shape
                times.append(float("inf"))
        best = candidates[min(range(len(candidates)), key=lambda i: times[i])]
        self.choices[k] = best
        self.timings[k] = dict(zip([str(c) for c in candidates], times))
        if self._path:
            with open(self._path, "w") as f:
                json.dump({kk: list(v) if isinstance(v, tuple) else v for kk, v in self.choices.items()}, f)
        return best


TUNER = Autotuner()
