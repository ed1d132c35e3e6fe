"""Float64 torch reference of the expected-value (mean-field) replay.

TEST INFRASTRUCTURE ONLY.  The window CSRs come from the C oracle
(orc.sorted_index / orc.schedule / orc.window_hits / orc.csr_i32, which
restate the reference's NCLS query with its hit cap and the per-step window
arithmetic of tool/gpu_cpu_temporal_sim.cu:859-991); the step is the
mean-field form of the geometric replay:

    e_i = scale * sum_j w_ij I_j,  P_i = 1 - exp(-beta s_i e_i)
    S' = S (1-P) + p_rs R [+ p_ir I if I->S]
    E' = E (1-p_ei) + S P                      (exposed state)
    I' = I (1-p_ir) + p_ei E  [+ S P without an exposed state]
    R' = R (1-p_rs) [+ p_ir I if I->R]
    incidence_t = sum_i S_i P_i

Gradients come from torch autograd in float64, and finite differences from
`central_difference`.
"""
import numpy as np
import torch

from . import orc


def window_csrs(start, end, u, v, n_nodes, start_time, step_size, window, n_steps, ncls_cap=True):
    """Per-step (row_ptr, col, weight, scale) with int32 contact-second weights."""
    ss, se, su, sv, perm, nl = orc.sorted_index(start, end, u, v)
    ws, we, sc, ts = orc.schedule(start_time, step_size, window, n_steps)
    out, cache = [], {}
    for t in range(n_steps):
        key = int(ws[t])
        if key not in cache:
            hits = orc.window_hits(ss, se, nl if ncls_cap else len(ss), int(ws[t]), int(we[t]))
            cache[key] = orc.csr_i32(ss, se, su, sv, hits, n_nodes, int(ws[t]), int(we[t]))
        rp, col, val = cache[key]
        out.append((rp, col, val, float(sc[t])))
    return out


def _torch_csrs(csrs):
    res = []
    for rp, col, val, scale in csrs:
        rows = torch.from_numpy(np.repeat(np.arange(len(rp) - 1), np.diff(rp)).astype(np.int64))
        res.append((rows, torch.from_numpy(col.astype(np.int64)), torch.from_numpy(val.astype(np.float64)),
                    scale))
    return res


def forward(csrs, x0, beta, sus, p_ei, p_ir, p_rs, has_exposed=True, ir_to_s=False):
    """x0: (4, N) float64 tensor.  Returns (incidence (T,), x_T (4, N))."""
    tcs = _torch_csrs(csrs)
    S, E, I, R = x0[0], x0[1], x0[2], x0[3]
    inc = []
    for rows, col, w, scale in tcs:
        e = torch.zeros_like(S).index_add(0, rows, w * I[col]) * scale
        s_i = sus if sus is not None else 1.0
        P = -torch.expm1(-beta * s_i * e)
        new = S * P
        f_ei = E * p_ei if has_exposed else torch.zeros_like(E)
        f_i, f_rs = I * p_ir, R * p_rs
        S2 = S * (1 - P) + f_rs + (f_i if ir_to_s else 0)
        E2 = E - f_ei + (new if has_exposed else 0)
        I2 = I - f_i + f_ei + (0 if has_exposed else new)
        R2 = R - f_rs + (0 if ir_to_s else f_i)
        S, E, I, R = S2, E2, I2, R2
        inc.append(new.sum())
    return torch.stack(inc) if inc else torch.zeros(0, dtype=x0.dtype), torch.stack([S, E, I, R])


def central_difference(fn, value, h_rel=1e-6):
    """d fn / d value by central differences in float64 (scalar value)."""
    h = h_rel * max(abs(float(value)), 1e-30)
    return (float(fn(value + h)) - float(fn(value - h))) / (2 * h)
