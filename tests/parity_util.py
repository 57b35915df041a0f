"""Shared drivers for the GPU parity tests: run the same sequence on the oracle
and on the engine, and record the measured discrepancies."""
import json
import os

import numpy as np

from bec_b200.engine import Engine
from oracle import oracle as O

LOG = os.environ.get("BEC_PARITY_LOG")
DUMP = os.environ.get("BEC_PARITY_DUMP")


def record(name, **vals):
    """Appends measured errors to $BEC_PARITY_LOG (JSON lines) when set."""
    if not LOG:
        return
    with open(LOG, "a") as f:
        f.write(json.dumps({"test": name, **{k: float(v) for k, v in vals.items()}}) + "\n")


def dump(name, **arrays):
    """Saves arrays to $BEC_PARITY_DUMP/<name>.npz when set (for offline error analysis)."""
    if not DUMP:
        return
    os.makedirs(DUMP, exist_ok=True)
    np.savez_compressed(os.path.join(DUMP, name + ".npz"), **arrays)


def rel_state_err(a, b):
    """max |a - b| / max |b| over both components."""
    return float(np.abs(a - b).max() / np.abs(b).max())


def moments_rel_err(m_eng, m_orc):
    """largest relative error of (na, nb, |s|) and absolute error of s relative to na + nb."""
    scale = m_orc[1] + m_orc[2]
    e = max(abs(m_eng[1] - m_orc[1]) / abs(m_orc[1]) if m_orc[1] else abs(m_eng[1]),
            abs(m_eng[2] - m_orc[2]) / abs(m_orc[2]) if m_orc[2] else abs(m_eng[2]))
    es = (abs(m_eng[3] - m_orc[3]) + abs(m_eng[4] - m_orc[4])) / scale
    return float(e), float(es)


def oracle_sequence(p, gs, steps, sample_every, noise=None, pi_pulse_step=-1, start=True):
    """Oracle: init, [start_evolution], steps with samples; returns (moments list, ensemble)."""
    e = O.OracleEnsemble(p)
    e.init(gs, noise)
    if start:
        e.start_evolution()
    out = []
    for i in range(1, steps + 1):
        e.evolve(1)
        if sample_every and i % sample_every == 0:
            out.append(e.moments())
        if i == pi_pulse_step:
            e.pulse(np.pi, 0.0)
    return np.array(out), e


def engine_sequence(p, gs, steps, sample_every, path, noise=None, pi_pulse_step=-1, start=True, use_run=True):
    eng = Engine([p], path=path)
    eng.init_group(0, gs, noise)
    if start:
        eng.start_evolution()
    if use_run:
        mom = eng.run(steps, sample_every=sample_every, pi_pulse_step=pi_pulse_step)[:, 0, :]
    else:
        out = []
        for i in range(1, steps + 1):
            eng.evolve(1)
            if sample_every and i % sample_every == 0:
                out.append(eng.moments()[0])
            if i == pi_pulse_step:
                eng.pulse(np.pi, 0.0)
        mom = np.array(out)
    return mom, eng
