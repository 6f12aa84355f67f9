"""Test-side restatement of Chaste's CellProperties (heart/src/postprocessing/CellProperties.cpp:55-312):
action-potential onsets, resting values and peaks, and APD at a given repolarisation percentage."""
import numpy as np


def apds(t, v, percentage=90.0, threshold=-30.0):
    t = np.asarray(t, float)
    v = np.asarray(v, float)
    rest_vals, onsets, peaks = [], [], []
    cur_rest, min_vel, flat = np.inf, np.inf, False
    cur_peak = -np.inf
    phase = 0
    prev_v, prev_t = v[0], t[0]
    for i in range(1, len(t)):
        vi, ti = v[i], t[i]
        vel = 0.0 if ti == prev_t else (vi - prev_v) / (ti - prev_t)
        if phase == 0:
            if abs(vel) <= min_vel and abs(vel) <= 1e-2:
                min_vel, cur_rest, flat = abs(vel), prev_v, True
            elif prev_v < cur_rest and not flat:
                cur_rest = prev_v
            if vi > threshold and prev_v <= threshold:
                rest_vals.append(cur_rest)
                min_vel, cur_rest = np.inf, np.inf
                onsets.append(prev_t + (ti - prev_t) / (vi - prev_v) * (threshold - prev_v))
                flat = False
                phase = 1
        if phase == 1:
            if vi > cur_peak:
                cur_peak = vi
            if vi < threshold and prev_v >= threshold:
                peaks.append(cur_peak)
                cur_peak = threshold
                phase = 0
        prev_v, prev_t = vi, ti
    out = []
    for k in range(len(peaks)):
        target = rest_vals[k] + 0.01 * (100 - percentage) * (peaks[k] - rest_vals[k])
        start_idx = int(np.searchsorted(t, onsets[k], side="left")) - 1
        start_time, start_index = None, None
        if target >= threshold:
            pv, pt = v[start_idx], t[start_idx]
            for j in range(start_idx + 1, len(t)):
                if v[j] > target:
                    start_time = pt + (target - pv) / (v[j] - pv) * (t[j] - pt)
                    start_index = j
                    break
                pt, pv = t[j], v[j]
        else:
            pv, pt = v[start_idx + 1], t[start_idx + 1]
            for j in range(start_idx, -1, -1):
                if v[j] < target:
                    start_time = pt + (target - pv) / (v[j] - pv) * (t[j] - pt)
                    start_index = j + 1
                    break
                pt, pv = t[j], v[j]
        if start_index is None:
            continue
        pv = v[start_index - 1]
        for j in range(start_index, len(t)):
            if v[j] < target:
                end = t[j - 1] + (target - pv) / (v[j] - pv) * (t[j] - t[j - 1])
                out.append(end - start_time)
                break
            pv = v[j]
    return out
