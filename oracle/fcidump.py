"""CPU restatement of ccq's FCIDUMP reader (test infrastructure only).

  * ``header``  <- ``get_fcidump`` (``src/parser.f90:260-313``) with
                   ``parse_key_val`` (``src/utils/utils.F90:416-462``)
  * ``load``    <- ``load_fcidump`` (``src/integrals.f90:93-210``) with the
                   stable ascending ``insertion_rank``
                   (``src/external/ranking.f90:84-141``)

Literal on purpose: the header of ``load`` ends at the first line whose
first token contains ``END`` (the list-directed ``read(unit, *) cur_line``),
records ``val i a j b`` are read list-directed (they may continue on the next
line; the rest of the line of the fifth value is dropped; the first record
that does not parse ends the read), every record is applied in file order.
Orbitals without an orbital-energy record get energy 0 (the reference leaves
that array uninitialised).  Only ``tests/`` use this module.
"""
from __future__ import annotations

import numpy as np


def _key_val(line, key):
    k = line.find(key)
    if k < 0:
        return None
    comma = line.find(',', k)
    if comma < 0:
        eq = line.find('=', k)
        val = line[eq + 1:]
    else:
        eq = line.find('=', k, comma)
        val = line[eq + 1:comma]
    return int(val.split()[0])


def header(path):
    """(NORB, NELEC); -1 when a key is absent."""
    norb = nelec = -1
    with open(path) as fh:
        for line in fh:
            if 'END' in line:
                break
            v = _key_val(line, 'NORB')
            if v is not None:
                norb = v
            v = _key_val(line, 'NELEC')
            if v is not None:
                nelec = v
    return norb, nelec


def _records(lines):
    k = 0
    while k < len(lines) and 'END' not in (lines[k].replace(',', ' ').split() or [''])[0]:
        k += 1
    k += 1
    recs = []
    while True:
        toks = []
        while len(toks) < 5 and k < len(lines):
            toks += lines[k].replace(',', ' ').split()
            k += 1
        if len(toks) < 5:
            break
        try:
            val = float(toks[0].replace('D', 'E').replace('d', 'e'))
            idx = [int(t) for t in toks[1:5]]
        except ValueError:
            break
        recs.append((val, *idx))
    return recs


def _insertion_rank(arr):
    """rank[k] = index of the k-th smallest value (1-based), stable."""
    rank = list(range(1, len(arr) + 1))
    for i in range(1, len(arr)):
        tmp = rank[i]
        j = i - 1
        while j >= 0 and arr[rank[j] - 1] > arr[tmp - 1]:
            rank[j + 1] = rank[j]
            j -= 1
        rank[j + 1] = tmp
    return rank


def load(path, norbs):
    """(e1int[i, a], e2int[i, j, a, b], E_nuc) as ``load_fcidump`` fills them."""
    with open(path) as fh:
        lines = fh.readlines()
    recs = _records(lines)
    eig = [0.0] * norbs
    for val, i, a, j, b in recs:
        if i != 0 and a + j + b == 0:
            eig[i - 1] = val
    rank = _insertion_rank(eig)
    inv = [0] * (norbs + 1)
    for idx in range(1, norbs + 1):
        inv[rank[idx - 1]] = idx
    e1 = np.zeros((norbs, norbs))
    e2 = np.zeros((norbs, norbs, norbs, norbs))
    hh = 0.0
    for val, i, a, j, b in recs:
        if i != 0 and a != 0 and j != 0 and b != 0:
            i, a, j, b = inv[i] - 1, inv[a] - 1, inv[j] - 1, inv[b] - 1
            for p, q, r, s in ((i, j, a, b), (j, i, b, a), (a, b, i, j), (b, a, j, i),
                               (a, j, i, b), (b, i, j, a), (i, b, a, j), (j, a, b, i)):
                e2[p, q, r, s] = val
        elif i != 0 and a != 0 and j + b == 0:
            i, a = inv[i] - 1, inv[a] - 1
            e1[i, a] = val
            e1[a, i] = val
        elif i + a + j + b == 0:
            hh = val
    return e1, e2, hh
