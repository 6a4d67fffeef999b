"""Independent numpy restatement of the reference's host baseliner, for the
tests only (a second reading of the reference code, separate from the
oracle's C++ one):

  * MultiStageFilter (src/basecaller/basecaller/traceAnalysis/
    HostMultiScaleBaseliner.h:110-149): lower = erode(w0, s0) -> dilate(w0),
    upper = dilate(w0, s0) -> erode(w0), then for every further scale i
    erode(wi, si) -> dilate(wi) on both, each stage a BlockFilterStage
    (BlockFilterStage.cpp:9-25) running in place over the first
    frames / nf entries with its own WindowBuffer (WindowBuffer.h);
  * extremumFilterHgw (TraceFilters.cpp:11-57): van Herk / Gil-Werman with
    the window's suffix extrema recomputed when the counter wraps, the
    holdover value kept across chunks, an initial window of w zeros;
  * EstimateBaseline, AddToBaselineStats and GetSmoothedBlEstimate
    (HostMultiScaleBaseliner.cpp:95-212) with the LaneArray conversions
    (float -> int16 by round-to-nearest-even, then 16-bit truncation; int16
    sums and differences wrap);
  * BaselinerStatAccumulator::AddSample / AddSampleBackground
    (dataTypes/BaselinerStatAccumulator.cpp:39-60, StatAccumulator.h:183-200,
    AutocorrAccumulator.cpp:29-39) for a fresh accumulator per chunk.

One lane (64 ZMWs) at a time, one chunk per call.
"""
import numpy as np

f32 = np.float32
LANE = 64


def wrap16(x):
    """int16 arithmetic result (wrapping)."""
    return np.asarray(x, np.int64).astype(np.int16)


def to_int16(xf):
    """LaneArray<float> -> LaneArray<short>: cvtps2dq (nearest-even; NaN and
    out-of-range give INT_MIN), then the low 16 bits."""
    r = np.rint(np.asarray(xf, np.float32).astype(np.float64))
    bad = ~np.isfinite(r) | (r >= 2.0 ** 31) | (r < -2.0 ** 31)
    r = np.where(bad, -2.0 ** 31, r).astype(np.int64)
    return (r & 0xffff).astype(np.uint16).view(np.int16)


class FilterStage:
    """BlockFilterStage with an ErodeHgw (min) or DilateHgw (max) filter."""

    def __init__(self, width, stride, nf, is_max):
        self.width, self.stride, self.nf, self.is_max = width, stride, nf, is_max
        self.window = [np.zeros(LANE, np.int16) for _ in range(width)]   # oldest first
        self.counter = 0
        self.holdover = np.zeros(LANE, np.int16)

    def _op(self, a, b):
        return np.maximum(a, b) if self.is_max else np.minimum(a, b)

    def __call__(self, data):
        n = len(data) // self.nf
        out = []
        s = self.holdover
        for i in range(0, n, self.stride):
            r = self.window
            if self.counter == 0:
                for j in range(self.width - 1, 0, -1):
                    r[j - 1] = self._op(r[j], r[j - 1])
                s = r[-1]
            else:
                s = self._op(s, r[-1])
            front = r[0]
            self.window = r[1:] + [data[i].copy()]
            self.counter = (self.counter + 1) % self.width
            out.append(self._op(s, front))
        self.holdover = s
        for k, v in enumerate(out):      # in place: output k after input k * stride was read
            data[k] = v


class MultiStageFilter:
    def __init__(self, strides, widths, upper):
        self.stages = [FilterStage(widths[0], strides[0], 1, upper),
                       FilterStage(widths[0], 1, strides[0], not upper)]
        for i in range(1, len(strides)):
            self.stages.append(FilterStage(widths[i], strides[i], strides[i - 1], False))
            self.stages.append(FilterStage(widths[i], 1, strides[i - 1] * strides[i], True))

    def __call__(self, data):
        for st in self.stages:
            st(data)
        return data


class LaneBaselinerRef:
    """HostMultiScaleBaseliner::LaneBaseliner for one lane."""

    def __init__(self, strides, widths, sigma_bias, mean_bias, scaler, pedestal, sigma_ema_alpha,
                 mean_ema_alpha, jump_tol_coeff=np.inf):
        self.lower = MultiStageFilter(strides, widths, False)
        self.upper = MultiStageFilter(strides, widths, True)
        self.stride = int(np.prod(strides))
        self.c_sigma, self.c_mean = f32(sigma_bias), f32(mean_bias)
        self.scaler, self.pedestal = f32(scaler), np.int16(pedestal)
        self.sigma_alpha, self.mean_alpha, self.jump = f32(sigma_ema_alpha), f32(mean_ema_alpha), f32(jump_tol_coeff)
        self.uema_sum = np.zeros(LANE, f32)
        self.uema_weight = np.zeros(LANE, f32)
        self.sigma_ema = np.full(LANE, f32(2.0))
        self.lat_data = np.zeros(LANE, np.int16)
        self.lat_raw = np.zeros(LANE, np.int16)
        self.lat_l = np.zeros(LANE, bool)
        self.lat_h1 = np.zeros(LANE, bool)
        self.lat_h2 = np.zeros(LANE, bool)

    def _smoothed_estimate(self, lower, upper):
        min_sigma = f32(.288675135)
        d = wrap16(upper.astype(np.int32) - lower.astype(np.int32)).astype(f32) / self.c_sigma
        sigma = np.where(d > min_sigma, d, min_sigma).astype(f32)          # SSE max: NaN -> second operand
        new_sigma = (self.sigma_alpha * self.sigma_ema + (f32(1) - self.sigma_alpha) * sigma).astype(f32)
        mid = wrap16(upper.astype(np.int32) + lower.astype(np.int32)).astype(f32)
        bl_est = (f32(0.5) * mid + self.c_mean * new_sigma).astype(f32)
        with np.errstate(divide="ignore", invalid="ignore"):
            mask = (self.uema_weight == 0) | ((bl_est - self.uema_sum / self.uema_weight) < self.jump * self.sigma_ema)
        new_weight = (self.mean_alpha * self.uema_weight + (f32(1) - self.mean_alpha)).astype(f32)
        new_sum = (self.mean_alpha * self.uema_sum + (f32(1) - self.mean_alpha) * bl_est).astype(f32)
        self.uema_weight = np.where(mask, new_weight, self.uema_weight)
        self.uema_sum = np.where(mask, new_sum, self.uema_sum)
        self.sigma_ema = np.where(mask, new_sigma, self.sigma_ema)
        return (self.uema_sum / self.uema_weight).astype(f32)

    def chunk(self, trace):
        """trace [F][64] int16 -> (baselined [F][64] int16, per-ZMW statistics)."""
        trace = np.ascontiguousarray(trace, np.int16)
        lower, upper = trace.copy(), trace.copy()
        self.lower(lower)
        self.upper(upper)
        out = np.zeros_like(trace)
        z = lambda: np.zeros(LANE, f32)
        st = {"bl_m0": z(), "bl_m1": z(), "bl_m2": z(), "raw_sum": z(), "bg_m0": z(), "bg_m1": z(), "bg_m2": z(),
              "all_m0": z(), "all_m1": z(), "all_m2": z(), "ac_m2": z(),
              "min": np.full(LANE, 32767, np.int16), "max": np.full(LANE, -32768, np.int16)}
        back = [np.zeros(LANE, f32) for _ in range(4)]
        n_added = 0
        for i in range(len(trace) // self.stride):
            lv = wrap16(lower[i].astype(np.int32) - self.pedestal)
            uv = wrap16(upper[i].astype(np.int32) - self.pedestal)
            sub = (self._smoothed_estimate(lv, uv) * self.scaler).astype(f32)
            for j in range(self.stride):
                f = i * self.stride + j
                rs = (wrap16(trace[f].astype(np.int32) - self.pedestal).astype(f32) * self.scaler).astype(f32)
                bls = to_int16(rs - sub)
                out[f] = bls
                raw = to_int16(rs)
                thr = (f32(4.5) * self.sigma_ema).astype(f32)
                hp1 = bls.astype(f32) < (thr * self.scaler).astype(f32)
                m = self.lat_h1 & self.lat_l & hp1
                self.lat_l = bls.astype(f32) < (thr * self.scaler).astype(f32)
                self.lat_h2 = self.lat_h1
                self.lat_h1 = hp1
                # AddSample(latRaw, latData, mask)
                v = self.lat_data.astype(f32)
                st["ac_m2"] = (st["ac_m2"] + back[n_added % 4] * v).astype(f32)
                back[n_added % 4] = v
                n_added += 1
                st["all_m0"] += f32(1)
                st["all_m1"] = (st["all_m1"] + v).astype(f32)
                st["all_m2"] = (st["all_m2"] + v * v).astype(f32)
                st["min"] = np.minimum(st["min"], self.lat_data)
                st["max"] = np.maximum(st["max"], self.lat_data)
                st["bl_m0"] = np.where(m, st["bl_m0"] + f32(1), st["bl_m0"])
                st["bl_m1"] = np.where(m, (st["bl_m1"] + v).astype(f32), st["bl_m1"])
                st["bl_m2"] = np.where(m, (st["bl_m2"] + v * v).astype(f32), st["bl_m2"])
                st["raw_sum"] = (st["raw_sum"] + np.where(m, self.lat_raw, 0).astype(f32)).astype(f32)
                self.lat_raw = raw
                self.lat_data = bls
            bg = to_int16(sub).astype(f32)
            st["bg_m0"] += f32(1)
            st["bg_m1"] = (st["bg_m1"] + bg).astype(f32)
            st["bg_m2"] = (st["bg_m2"] + bg * bg).astype(f32)
        return out, st
