"""Round checkpoints: stop an inference after any round and continue it later
with the same trajectory, bit for bit.

The reference can restart an interrupted run from its last run directory
(Mi3.py:373-421, `--finish`): it reloads that round's starting couplings and
the sequences it wrote, and runs the round again; the walkers' RNG streams
and the site list start over, so the continuation differs from the run that
was interrupted.  A checkpoint here holds everything the next round depends
on -- per device the walkers (packed sequence words), the MWC64X states, the
site list with its read offset and the host MT19937 state that refills it;
and for the round loop the couplings, the step counter, the Newton step
budget and SSR memory, the history and the reseed generator -- so a run
continued from it takes exactly the steps the uninterrupted run would have
taken.  Written atomically (temporary file + rename) after each round.
"""
import os
import pickle
from pathlib import Path

import numpy as np

FORMAT = 1

_PARAM_KEYS = ('newtonSteps', 'max_newtonSteps', 'last_ssr', 'min_ssr', 'history', 'seedseq')


def rank_path(path, gpus):
    """The checkpoint file of this process: `path` itself, or, when the
    devices are spread over ranks (distributed.RankNode, one device per
    rank), `path` with '.rank<r>' appended -- each rank checkpoints its own
    walkers and resumes from its own file."""
    path = Path(path)
    world = getattr(gpus, 'world', 1)
    return path if world <= 1 else path.with_name(f"{path.name}.rank{gpus.rank}")


def device_state(gpu):
    """Host copy of one device's sampling state."""
    get = getattr(gpu, 'state_dict', None)
    if get is None:
        raise TypeError(f"{type(gpu).__name__} has no state_dict()")
    return get()


def save(path, gpus, param, next_run, Jstep, J, rng, seqs=None, es=None):
    """Write the state after a finished round; `next_run` is the index of the
    round to run next.  J is the host couplings (None when they live on the
    devices, in which case they are read from the head device)."""
    if J is None:
        J = gpus.head_gpu.readBufs('J')[0]
    state = {
        'format': FORMAT,
        'next_run': int(next_run),
        'Jstep': int(Jstep),
        'J': np.asarray(J, dtype='<f4').copy(),
        'param': {k: param.get(k) for k in _PARAM_KEYS},
        'reseed_rng': rng.get_state(),
        'seqs': None if seqs is None else np.asarray(seqs),
        'es': None if es is None else np.asarray(es),
        'devices': [device_state(g) for g in gpus.gpus],
        'shape': (int(param.L), int(param.q), int(gpus.nwalkers)),
    }
    path = rank_path(path, gpus)
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_name(f"{path.name}.{os.getpid()}.tmp")
    with open(tmp, 'wb') as f:
        pickle.dump(state, f, protocol=pickle.HIGHEST_PROTOCOL)
    os.replace(tmp, path)


def load(path):
    with open(path, 'rb') as f:
        state = pickle.load(f)
    if state.get('format') != FORMAT:
        raise ValueError(f"{path}: unsupported checkpoint format {state.get('format')}")
    return state


def restore(state, gpus, param, rng):
    """Put a loaded checkpoint back into the devices, `param` and the reseed
    generator; returns (start_run, Jstep, J, seqs, es)."""
    L, q, n = state['shape']
    if (L, q, n) != (int(param.L), int(param.q), int(gpus.nwalkers)):
        raise ValueError(f"checkpoint is for L={L} q={q} walkers={n}, not "
                         f"L={param.L} q={param.q} walkers={gpus.nwalkers}")
    if len(state['devices']) != len(gpus.gpus):
        raise ValueError("checkpoint was written by a different number of devices")
    for g, d in zip(gpus.gpus, state['devices']):
        g.load_state_dict(d)
    for k, v in state['param'].items():
        param[k] = v
    rng.set_state(state['reseed_rng'])
    return state['next_run'], state['Jstep'], state['J'], state['seqs'], state['es']
