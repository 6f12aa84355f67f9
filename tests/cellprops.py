"""Test-side restatement of Chaste's CellProperties (heart/src/postprocessing/CellProperties.cpp)
and of the per-node maps PostProcessingWriter writes from it
(heart/src/postprocessing/PostProcessingWriter.cpp:226-345,
heart/src/postprocessing/PropagationPropertiesCalculator.cpp:60-160, 226-280)."""
import numpy as np

UNSET = None


class NoAp(Exception):
    pass


def calculate_properties(t, v, threshold=-30.0):
    """CellProperties::CalculateProperties (CellProperties.cpp:55-220)."""
    t = np.asarray(t, float)
    v = np.asarray(v, float)
    p = dict(onsets=[], rest=[], peaks=[], peak_times=[], max_up=[], t_max_up=[], unfinished=False)
    max_up, t_up = -np.finfo(float).max, 0.0
    cur_rest, cur_peak, cur_peak_t = np.finfo(float).max, -np.finfo(float).max, -np.finfo(float).max
    min_vel = np.finfo(float).max
    flat = False
    phase = 0
    prev_v, prev_t = v[0], t[0]
    for i in range(1, len(t)):
        vi, ti = v[i], t[i]
        vel = 0.0 if ti == prev_t else (vi - prev_v) / (ti - prev_t)
        if vel >= max_up:
            max_up, t_up = vel, ti
        if phase == 0:
            if abs(vel) <= min_vel and abs(vel) <= 1e-2:
                min_vel, cur_rest, flat = abs(vel), prev_v, True
            elif prev_v < cur_rest and not flat:
                cur_rest = prev_v
            if vi > threshold and prev_v <= threshold:
                p["rest"].append(cur_rest)
                min_vel, cur_rest = np.finfo(float).max, np.finfo(float).max
                p["onsets"].append(prev_t + (ti - prev_t) / (vi - prev_v) * (threshold - prev_v))
                flat = False
                phase = 1
        if phase == 1:
            if vi > cur_peak:
                cur_peak, cur_peak_t = vi, ti
            if vi < threshold and prev_v >= threshold:
                p["peaks"].append(cur_peak)
                p["peak_times"].append(cur_peak_t)
                cur_peak, cur_peak_t = threshold, -np.finfo(float).max
                p["max_up"].append(max_up)
                max_up = -np.finfo(float).max
                p["t_max_up"].append(t_up)
                t_up = 0.0
                phase = 0
        prev_v, prev_t = vi, ti
    if len(p["onsets"]) > len(p["max_up"]):
        p["max_up"].append(max_up)
        p["peaks"].append(cur_peak)
        p["peak_times"].append(cur_peak_t)
        p["t_max_up"].append(t_up)
        p["unfinished"] = True
    return p


def action_potential_durations(t, v, p, percentage=90.0, threshold=-30.0):
    """CellProperties::CalculateActionPotentialDurations (CellProperties.cpp:222-330),
    including the start and end times carried from one action potential to the next."""
    t = np.asarray(t, float)
    v = np.asarray(v, float)
    if not p["onsets"]:
        raise NoAp("AP did not occur, never exceeded threshold voltage.")
    out = []
    start_time, end_time, start_index = UNSET, UNSET, UNSET
    for k in range(len(p["peaks"])):
        target = p["rest"][k] + 0.01 * (100 - percentage) * (p["peaks"][k] - p["rest"][k])
        sti = int(np.searchsorted(t, p["onsets"][k], side="left")) - 1
        if target >= threshold:
            pv, pt = v[sti], t[sti]
            for j in range(sti + 1, len(t)):
                if v[j] > target:
                    start_time = pt + ((target - pv) / (v[j] - pv)) * (t[j] - pt)
                    start_index = j
                    break
                pt, pv = t[j], v[j]
        else:
            pv, pt = v[sti + 1], t[sti + 1]
            for j in range(sti, -1, -1):
                if v[j] < target:
                    start_time = pt + ((target - pv) / (v[j] - pv)) * (t[j] - pt)
                    start_index = j + 1
                    break
                pt, pv = t[j], v[j]
        if end_time is not UNSET and start_time is not UNSET and start_time < end_time:
            continue
        if start_index is not UNSET:
            pv = v[start_index - 1]
            for j in range(start_index, len(t)):
                if v[j] < target:
                    end_time = t[j - 1] + ((target - pv) / (v[j] - pv)) * (t[j] - t[j - 1])
                    out.append(end_time - start_time)
                    break
                pv = v[j]
    if not out:
        raise NoAp("No full action potential was recorded")
    return out


def apds(t, v, percentage=90.0, threshold=-30.0):
    """APDs of one trace (an empty list when Chaste would raise)."""
    try:
        return action_potential_durations(t, v, calculate_properties(t, v, threshold), percentage, threshold)
    except NoAp:
        return []


def node_maps(t, frames, percentage=90.0, threshold=-30.0):
    """Per-node lists as PostProcessingWriter writes them: APD map, upstroke-time map and
    maximum-upstroke-velocity map, [0] where CellProperties raises."""
    apd_map, up_t, up_v = [], [], []
    for i in range(frames.shape[1]):
        p = calculate_properties(t, frames[:, i], threshold)
        try:
            apd_map.append(action_potential_durations(t, frames[:, i], p, percentage, threshold))
        except NoAp:
            apd_map.append([0.0])
        up_t.append(p["t_max_up"] if p["max_up"] else [0.0])
        up_v.append(p["max_up"] if p["max_up"] else [0.0])
    return apd_map, up_t, up_v


def conduction_velocities(up_t_near, up_t_far, distance, same_node):
    """PropagationPropertiesCalculator::CalculateAllConductionVelocities (:226-280) on
    upstroke-time lists ([0] where either node has none)."""
    if not up_t_near or not up_t_far:
        return [0.0]
    n = min(len(up_t_near), len(up_t_far))
    if same_node:
        return [0.0] * n
    out = []
    for i in range(n):
        dt = up_t_far[i] - up_t_near[i]
        out.append(0.0 if abs(dt) < 1e-8 else distance / dt)
    return out
