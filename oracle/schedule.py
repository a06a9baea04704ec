"""Restatement of the reference's host-side path control. TEST INFRASTRUCTURE ONLY: tests/ use it
to check the library's nrrs_ubs_* and nrrs_train_schedule_* entry points, never the product.

In banbao990/NRRS-Code (NRRSPathTracer):
  UBS search and use          src/render/nrrs/integrator.h:324-405, integrator.cpp:2787-2889
  isInferMode                 src/render/nrrs/integrator.h:67-71
  factor source per depth     src/render/nrrs/integrator.cpp:1088-1090
  autoTrainControl            src/render/nrrs/integrator.cpp:2659-2736
Float fields are float32, as in the reference; the frame clock is the caller's.
"""
from __future__ import annotations

import numpy as np

F = np.float32
COUNT = 3
FIXED_RR, ADN, NRRS = 0, 1, 2
FACTOR_ADRRS, FACTOR_RRSNET = 2, 3


class UBSRef:
    def __init__(self, max_depth: int = 6, error_eval_seconds: float = 0.17e-3):
        self.max_depth = max_depth
        self.eval = error_eval_seconds
        self.search = False
        self.use_best = False
        self.array = [0] * 64                  # zero-filled, integrator.cpp:42-45
        self.best_eff = F(-1.0)
        self.state, self.mod, self.last_state = -1, -1, -1
        self.max_state, self.best_state, self.cnt = 0, 0, 0
        self.timer = False
        self.last_error, self.last_dt = F(-1.0), F(-1.0)
        self.last_time = 0.0

    def begin(self):                           # UBSResetAndBeginSearch, integrator.h:376-389
        self.best_eff = F(0.0)
        self.last_error, self.last_dt = F(-1.0), F(-1.0)
        self.search, self.use_best = True, False
        self.state = self.mod = self.last_state = -1
        self.max_state = int(F(3.0 ** self.max_depth))   # (int) pow(3.0f, (float) mMaxDepth)

    def end(self):                             # UBSEndSearch, integrator.h:391-405
        self.timer = False
        self.search = False
        s = self.best_state
        for i in range(self.max_depth):
            self.array[i] = s % COUNT
            s //= COUNT

    def next_state(self) -> bool:              # UBSNextState, integrator.cpp:2798-2820
        if not self.search:
            return False
        if self.state < self.max_state:
            self.last_state = self.state
            if self.state == 0:
                self.cnt = 0
            self.mod += 1
            if self.mod == 729:
                self.cnt += 1
                self.state = self.best_state
            self.state += 729 ** self.cnt
            return True
        self.end()
        return False

    def analyse(self, now: float, err_sum: float, res: int):   # UBSAnalyseFrame, :2822-2889
        if not self.search:
            return
        if not self.timer:
            self.begin()
            self.timer = True
            self.last_time = now
            return
        dt = F(now - self.last_time)
        self.last_time = now
        if self.last_error < 0:
            keep = self.last_state
            self.begin()
            self.last_state = keep
        elif self.last_state >= 0:
            self.last_dt = F(self.last_dt - F(self.eval))
            eff = F(F(res) / F(self.last_dt * self.last_error))
            if eff > self.best_eff:             # UBSRecordEfficiency, :2787-2796
                self.best_eff = eff
                self.best_state = self.last_state
        self.last_dt = dt
        self.last_error = F(err_sum)

    def digit(self, depth: int) -> int:
        return (self.state // COUNT ** depth) % COUNT

    def strategy(self, depth: int) -> int:
        if self.search:
            return self.digit(depth)
        if self.use_best:
            return self.array[depth]
        return -1

    def need_infer(self, depth, enable_rrs, cmin, cmax, max_rrs_depth, use_net):
        need = True
        if self.use_best:
            need = self.array[depth] != FIXED_RR
        elif self.search:
            need = self.digit(depth) != FIXED_RR
        infer = bool(enable_rrs) and F(cmin) < F(cmax) and depth <= max_rrs_depth and need
        net = bool(use_net)
        if self.search:
            net = self.digit(depth) == NRRS
        elif self.use_best:
            net = self.array[depth] == NRRS
        return infer, FACTOR_RRSNET if net else FACTOR_ADRRS

    def set_best(self, digits: str):           # UBSUpdateAccordingArrayChar, integrator.h:364-374
        for i in range(self.max_depth):
            n = ord(digits[i]) - ord("0") if i < len(digits) else -1
            self.array[i] = n if 0 <= n < COUNT else FIXED_RR
        self.use_best = True


class ScheduleRef:                              # autoTrainControl, integrator.cpp:2659-2736
    def __init__(self, durations):
        self.end = [0.0] * 5
        for i in range(1, 5):
            self.end[i] = self.end[i - 1] + durations[i - 1]
        self.state = -1
        self.o = dict(state=0, step=0, enable_rrs=0, use_net_output_rrs=0, stop_training=0,
                      request_exit=0, seconds_per_frame=0.0)
        self.count = 100
        self.start = 0.0

    def tick(self, elapsed: float, now: float) -> dict:
        o = self.o
        over = lambda st: elapsed > self.end[st + 1]  # noqa: E731
        if self.state == -1:
            self.state, o["enable_rrs"], o["step"] = 0, 0, 0
        if self.state == 0 and over(0):
            self.state, o["enable_rrs"], o["step"] = 1, 0, 1
        if self.state == 1 and over(1):
            self.state, o["enable_rrs"], o["use_net_output_rrs"], o["step"] = 2, 1, 0, 2
        if self.state == 2 and over(2):
            self.state, o["use_net_output_rrs"], o["step"] = 3, 1, 3
        if self.state == 3 and over(3):
            o["stop_training"] = 1
            if self.count == 100:
                self.start = now
            self.count -= 1
            if self.count < 0:
                o["seconds_per_frame"] = (now - self.start) / 100.0
                self.state = 4
        if self.state == 4:
            o["request_exit"] = 1
        o["state"] = self.state
        return dict(o)
