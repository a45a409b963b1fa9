"""Matrix / vector dump files of hecmw_matrix_dump (hecmw1/src/solver/matrix/hecmw_matrix_dump.f90).

`!SOLVER, DUMPTYPE=MM|CSR|BSR` makes hecmw_solve_iterative write, before the solve,
the matrix of the call (`dump_matrix_<call>_<rank>.mm|.csr|.bsr`) and its right-hand
side (`.rhs`), and after it the solution (`.sol`); `DUMPEXIT=YES` stops the program
after the matrix dump.  The formats (:30-367):

  .mm   MatrixMarket coordinate, scalar entries (3x3 blocks expanded), row-major
        within each block row: L blocks, D, U blocks (:62-124)
  .csr  scalar CSR: header, index(0:nrow), item(1:nnz) 1-based, value(1:nnz) (:126-233)
  .bsr  block CSR: header, index(0:nrow), item(1:nnz) 1-based block ids, then the
        nnz 3x3 blocks, one value per line, row-major (:235-307)
  .rhs / .sol  one value per line, 3*NP values (:309-367)

Values are written with the Fortran edit descriptor e20.12e3 (`fortran_e`); the
readers accept any float syntax.  Readers return a HecMatrix (Iarray/Rarray at the
hecmw defaults), so a matrix dumped by fistr1 can be handed to the solver directly.
"""
import math
import os

import numpy as np

from .matrix import HecMatrix, IDX_I_DUMP, IDX_I_DUMP_EXIT

DUMP_NONE, DUMP_MM, DUMP_CSR, DUMP_BSR = 0, 1, 2, 3
_EXT = {DUMP_MM: ".mm", DUMP_CSR: ".csr", DUMP_BSR: ".bsr"}


def fortran_e(v):
    """v in the Fortran edit descriptor e20.12e3: ' 0.dddddddddddd E+xxx' (20 chars)."""
    v = float(v)
    if v != v:
        return "NaN".rjust(20)
    if math.isinf(v):
        return ("-Infinity" if v < 0 else "Infinity").rjust(20)
    sign = "-" if math.copysign(1.0, v) < 0 else " "
    if v == 0.0:
        return sign + "0.000000000000E+000"
    mant, exp = ("%.11e" % abs(v)).split("e")
    e = int(exp) + 1
    return sign + "0." + mant.replace(".", "") + "E" + ("-" if e < 0 else "+") + "%03d" % abs(e)


def _blocks_rows(m):
    """Per block row: (L item/blocks, D block, U item/blocks), 1-based items."""
    D = m.D.reshape(-1, 9)
    AL = m.AL.reshape(-1, 9)
    AU = m.AU.reshape(-1, 9)
    for i in range(m.NP):
        lo = range(m.indexL[i], m.indexL[i + 1])
        up = range(m.indexU[i], m.indexU[i + 1])
        yield i, [(int(m.itemL[k]), AL[k]) for k in lo] + [(i + 1, D[i])] + [(int(m.itemU[k]), AU[k]) for k in up]


def write_bsr(m, path):
    """hecmw_mat_dump_bsr (:235-307)."""
    nnz = m.NP + int(m.indexL[m.NP]) + int(m.indexU[m.NP])
    with open(path, "w") as f:
        f.write("%%Block-CSR matrix real general\n")
        f.write("% nrow ncol nnonzero ndof\n")
        f.write("%d %d %d %d\n" % (m.NP, m.NP, nnz, 3))
        f.write("% index(0:nrow)\n")
        idx = 0
        f.write("0\n")
        for i in range(m.NP):
            idx += int(m.indexL[i + 1] - m.indexL[i]) + 1 + int(m.indexU[i + 1] - m.indexU[i])
            f.write("%d\n" % idx)
        rows = list(_blocks_rows(m))
        f.write("% item(1:nnonzero)\n")
        for _, blocks in rows:
            for j, _b in blocks:
                f.write("%d\n" % j)
        f.write("% value(1:nnonzero*ndof*ndof)\n")
        for _, blocks in rows:
            for _j, b in blocks:
                for v in b:
                    f.write(fortran_e(v) + "\n")


def write_csr(m, path):
    """hecmw_mat_dump_csr (:126-233): scalar rows, each block row's 3 rows in turn."""
    rows = list(_blocks_rows(m))
    nnz = 9 * sum(len(b) for _, b in rows)
    with open(path, "w") as f:
        f.write("%%CSR matrix real general\n")
        f.write("% nrow ncol nnonzero\n")
        f.write("%d %d %d\n" % (3 * m.NP, 3 * m.NP, nnz))
        f.write("% index(0:nrow)\n")
        f.write("0\n")
        idx = 0
        for _, blocks in rows:
            for _a in range(3):
                idx += 3 * len(blocks)
                f.write("%d\n" % idx)
        f.write("% item(1:nnonzero)\n")
        for _, blocks in rows:
            for _a in range(3):
                for j, _b in blocks:
                    for c in range(3):
                        f.write("%d\n" % (3 * (j - 1) + c + 1))
        f.write("% value(1:nnonzero)\n")
        for _, blocks in rows:
            for a in range(3):
                for _j, b in blocks:
                    for c in range(3):
                        f.write(fortran_e(b[3 * a + c]) + "\n")


def write_mm(m, path):
    """hecmw_mat_dump_mm (:62-124)."""
    rows = list(_blocks_rows(m))
    nnz = 9 * sum(len(b) for _, b in rows)
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write("%d %d %d\n" % (3 * m.NP, 3 * m.NP, nnz))
        for i, blocks in rows:
            for a in range(3):
                for j, b in blocks:
                    for c in range(3):
                        f.write("%d %d %s\n" % (3 * i + a + 1, 3 * (j - 1) + c + 1, fortran_e(b[3 * a + c])))


def write_vector(v, path):
    """hecmw_mat_dump_rhs / _solution (:309-367)."""
    with open(path, "w") as f:
        for x in np.asarray(v, dtype=np.float64):
            f.write(fortran_e(x) + "\n")


def read_vector(path):
    return np.array([float(t) for t in open(path).read().split()], dtype=np.float64)


def _data_lines(path):
    for line in open(path):
        t = line.strip()
        if t and not t.startswith("%"):
            yield t


def _from_block_rows(n, items, blocks):
    """HecMatrix from per-row lists of (1-based block column, 9 values)."""
    indexL, indexU, itemL, itemU, AL, AU = [0], [0], [], [], [], []
    D = np.zeros((n, 9))
    for i in range(n):
        for j, b in zip(items[i], blocks[i]):
            if j < i + 1:
                itemL.append(j)
                AL.append(b)
            elif j == i + 1:
                D[i] = b
            else:
                itemU.append(j)
                AU.append(b)
        indexL.append(len(itemL))
        indexU.append(len(itemU))
    # keep the arrays non-empty (as HecMatrix.empty does); indexL/indexU say how many count
    for items_, vals_ in ((itemL, AL), (itemU, AU)):
        if not items_:
            items_.append(0)
            vals_.append(np.zeros(9))
    m = HecMatrix(n, n, np.array(indexL, np.int32), np.array(itemL, np.int32), np.array(indexU, np.int32),
                  np.array(itemU, np.int32), D.reshape(-1),
                  np.array(AL, np.float64).reshape(-1), np.array(AU, np.float64).reshape(-1))
    for arr, idx in ((m.itemL, m.indexL), (m.itemU, m.indexU)):
        for i in range(n):
            seg = arr[idx[i]:idx[i + 1]]
            if np.any(np.diff(seg) <= 0):
                raise ValueError("dump: block columns of row %d are not ascending" % (i + 1))
    return m


def read_bsr(path):
    """A HecMatrix from a .bsr dump (ndof 3)."""
    it = _data_lines(path)
    nrow, ncol, nnz, ndof = (int(t) for t in next(it).split())
    if ndof != 3 or nrow != ncol:
        raise ValueError("dump: a square matrix of 3x3 blocks is expected")
    index = [int(next(it)) for _ in range(nrow + 1)]
    item = [int(next(it)) for _ in range(nnz)]
    vals = np.array([float(next(it)) for _ in range(9 * nnz)]).reshape(nnz, 9)
    items = [item[index[i]:index[i + 1]] for i in range(nrow)]
    blocks = [vals[index[i]:index[i + 1]] for i in range(nrow)]
    return _from_block_rows(nrow, items, blocks)


def _from_scalar(nrow, entries):
    """HecMatrix from scalar (row, col, value), 0-based, 3 DOF per node."""
    n = nrow // 3
    rows = [dict() for _ in range(n)]
    for r, c, v in entries:
        blk = rows[r // 3].setdefault(c // 3 + 1, np.zeros(9))
        blk[3 * (r % 3) + c % 3] = v
    items = [sorted(d) for d in rows]
    blocks = [[rows[i][j] for j in items[i]] for i in range(n)]
    return _from_block_rows(n, items, blocks)


def read_csr(path):
    it = _data_lines(path)
    nrow, ncol, nnz = (int(t) for t in next(it).split())
    index = [int(next(it)) for _ in range(nrow + 1)]
    item = [int(next(it)) for _ in range(nnz)]
    vals = [float(next(it)) for _ in range(nnz)]
    ent = [(r, item[k] - 1, vals[k]) for r in range(nrow) for k in range(index[r], index[r + 1])]
    return _from_scalar(nrow, ent)


def read_mm(path):
    it = _data_lines(path)
    nrow, ncol, nnz = (int(t) for t in next(it).split())
    ent = []
    for _ in range(nnz):
        r, c, v = next(it).split()
        ent.append((int(r) - 1, int(c) - 1, float(v)))
    return _from_scalar(nrow, ent)


READERS = {".bsr": read_bsr, ".csr": read_csr, ".mm": read_mm}


def read_matrix(path):
    """A HecMatrix from any of the three matrix dumps (by extension)."""
    return READERS[os.path.splitext(path)[1]](path)


class Dumper:
    """The dump calls of hecmw_solve_iterative for one process (NumCall counts calls,
    `rank` is the domain's rank); files go to `directory`."""

    def __init__(self, directory=".", rank=0):
        self.directory = directory
        self.rank = rank
        self.num_call = 0

    def _name(self, ext):
        return os.path.join(self.directory, "dump_matrix_%d_%d%s" % (self.num_call, self.rank, ext))

    def dump(self, m):
        """hecmw_mat_dump (:30-49): matrix + right-hand side; DUMPEXIT stops the program."""
        self.num_call += 1
        kind = int(m.Iarray[IDX_I_DUMP - 1])
        if kind == DUMP_NONE:
            return
        {DUMP_MM: write_mm, DUMP_CSR: write_csr, DUMP_BSR: write_bsr}[kind](m, self._name(_EXT[kind]))
        write_vector(m.B[:3 * m.NP], self._name(".rhs"))
        if int(m.Iarray[IDX_I_DUMP_EXIT - 1]) != 0:
            raise SystemExit("Exiting program after dumping matrix")

    def dump_solution(self, m):
        """hecmw_mat_dump_solution (:339-367)."""
        if int(m.Iarray[IDX_I_DUMP - 1]) == DUMP_NONE:
            return
        write_vector(m.X[:3 * m.NP], self._name(".sol"))
