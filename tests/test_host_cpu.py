"""CPU tests of the host side: the C ABI library loads and exports every
entry point its headers declare, the Python face validates its arguments as
lng_GAUSS_SEIDEL_SOLVER_new does (lng.c:4243-4345), and the multi-GPU
plumbing of bench.py (replicas, slowest-rank time) runs on two gloo ranks."""
import ctypes as C
import os
import re
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, 'include', h) for h in ('solfec_b200.h', 'b2_device.h')]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r'/\*.*?\*/', '', open(h).read(), flags=re.S)
        for m in re.finditer(r'\b((?:b2gs|b2dev)_[a-z0-9_]+)\s*\(', text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from solfec_b200 import _lib
    path = _lib.build()
    L = C.CDLL(path)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert set(declared_functions()) <= set(_lib.exported_symbols()), 'Python binding lacks signatures'
    out = subprocess.run(['nm', '-D', '--defined-only', path], capture_output=True, text=True).stdout
    for n in declared_functions():
        assert re.search(r' T %s$' % n, out, flags=re.M), n


def test_solver_parameters_and_strings():
    from solfec_b200 import GAUSS_SEIDEL_SOLVER
    gs = GAUSS_SEIDEL_SOLVER(1e-4, 1000)
    assert gs.failure == 'FAILURE_CONTINUE' and gs.diagsolver == 'SEMISMOOTH_NEWTON'
    assert gs.error == 'OK' and gs.reverse == 'OFF' and gs.variant == 'FULL' and gs.iters == 0
    assert gs.meritval == 1.0 and gs.nomerit
    gs.reverse = 'ON'
    assert gs.reverse == 'ON'
    gs.variant = 'MIDDLE_JACOBI'
    assert gs.variant == 'MIDDLE_JACOBI'
    assert GAUSS_SEIDEL_SOLVER(1e-3, 10, 1e-3, 'EXIT', diagsolver='DE_SAXCE_FENG').diagsolver == 'DE_SAXCE_FENG'
    for bad in (dict(epsilon=0, maxiter=10), dict(epsilon=1e-3, maxiter=0), dict(epsilon=1e-3, maxiter=5, meritval=-1),
                dict(epsilon=1e-3, maxiter=5, failure='STOP'), dict(epsilon=1e-3, maxiter=5, diagsolver='DIAGONAL'),
                dict(epsilon=1e-3, maxiter=5, failure='CALLBACK')):
        with pytest.raises(ValueError):
            GAUSS_SEIDEL_SOLVER(**bad)
    assert gs.write_state().startswith('GSITERS 0')


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


WORKER = r'''
import os, sys
sys.path.insert(0, %(root)r)
import torch.distributed as dist
import bench
dist.init_process_group('gloo', init_method='env://')
r = dist.get_rank()
t = bench.max_over_ranks(10.0 + 5.0 * r)
seeds = [None, None]
dist.all_gather_object(seeds, bench.replica_seed(r))
print('rank', r, 'max', t, 'seeds', seeds)
assert t == 15.0 and seeds == [3, 4]
dist.barrier()
dist.destroy_process_group()
'''


def test_replica_timing_on_two_gloo_ranks():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(r), WORLD_SIZE='2')
        procs.append(subprocess.Popen([sys.executable, '-c', WORKER % {'root': ROOT}], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            outs.append(p.communicate(timeout=120)[0])
        except subprocess.TimeoutExpired:
            p.kill()
            outs.append(p.communicate()[0])
    assert all(p.returncode == 0 for p in procs), outs
    assert 'max 15.0' in outs[0] and 'max 15.0' in outs[1]
