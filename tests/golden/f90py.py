"""Mechanical Fortran-90 + MPI to Python translation, with an in-process MPI.

Used by make_golden.py to execute the reference programs themselves
(natural-convection_{2,3}dim_{mono,block}.f90 of zzhao0930/MPI-Multi-Process-Version)
so that their outputs pin the CPU oracle.  Test infrastructure only.

Scope: the Fortran subset those four programs use -- one module of globals,
subroutines, one pure function, the main program; integer/real(8)/logical
scalars and arrays with explicit lower bounds, allocatable and automatic
arrays, `data` statements, `parameter`s, do / do while / if chains, array
element, section and whole-array assignment, array constructors, the
intrinsics dble, sqrt, dsqrt, erf, mod, abs, min, max, and the MPI routines
they call.  Output statements are dropped, except, with `with_output`, the
formatted writes to numbered units (open / write with a format label or
list-directed / format statements), which render through f90fmt.py into
S._io[unit] -- the reference's Tecplot writer output_ASCII; character
variables are dropped.

Arithmetic follows gfortran -O2 on x86-64: IEEE double, operands evaluated
left to right inside the parentheses the source gives, no contraction;
x**2 and x**2.0d0 become x*x and x**3 becomes (x*x)*x (GCC's powi expansion);
real literals without a d exponent are single precision (rounded through
float32), as Fortran requires.

The MPI emulation runs every rank as a thread over one shared "world":
point-to-point sends are buffered, receives block, collectives exchange
through a barrier; MPI_PROC_NULL partners are no-ops; Cartesian topologies are
row-major as in the MPI standard (MPI_Dims_create balances the factors).
MPI_Allreduce sums in rank order.
"""
from __future__ import annotations

import math
import re
import struct
import threading
import time
from collections import defaultdict, deque

# ---------------------------------------------------------------------------
# runtime support
# ---------------------------------------------------------------------------


def f32(x: float) -> float:
    return struct.unpack("f", struct.pack("f", x))[0]


class FArray:
    """A Fortran array: explicit bounds, column-major flat storage (a list)."""

    __slots__ = ("lb", "ext", "data", "kind")

    def __init__(self, bounds, kind="real"):
        self.lb = [int(b[0]) for b in bounds]
        self.ext = [int(b[1]) - int(b[0]) + 1 for b in bounds]
        n = 1
        for e in self.ext:
            n *= max(e, 0)
        self.kind = kind
        self.data = [0.0 if kind == "real" else (False if kind == "logical" else 0)] * n

    def off(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        o, mul = 0, 1
        for d, i in enumerate(idx):
            k = i - self.lb[d]
            if k < 0 or k >= self.ext[d]:
                raise IndexError(f"index {idx} out of bounds lb={self.lb} ext={self.ext}")
            o += k * mul
            mul *= self.ext[d]
        return o

    def __getitem__(self, idx):
        return self.data[self.off(idx)]

    def __setitem__(self, idx, v):
        self.data[self.off(idx)] = v

    def dim_range(self, d):
        return range(self.lb[d], self.lb[d] + self.ext[d])


class Stop(Exception):
    pass


PROC_NULL = -2


class World:
    def __init__(self, n):
        self.n = n
        self.barrier = threading.Barrier(n, timeout=600)
        self.cv = threading.Condition()
        self.slots = {}
        self.queues = defaultdict(deque)
        self.failed = False
        self.t0 = time.perf_counter()
        self.dims = None


class Comm:
    """The MPI routines the reference calls, for one rank."""

    def __init__(self, world: World, rank: int):
        self.w, self.rank, self.size, self.seq = world, rank, world.n, 0

    # --- environment
    def wtime(self):
        return time.perf_counter() - self.w.t0

    def barrier(self):
        self.w.barrier.wait()

    def _exchange(self, value):
        w, key = self.w, self.seq
        self.seq += 1
        with w.cv:
            w.slots[(key, self.rank)] = value
        w.barrier.wait()
        vals = [w.slots[(key, r)] for r in range(w.n)]
        w.barrier.wait()
        if self.rank == 0:
            with w.cv:
                for r in range(w.n):
                    del w.slots[(key, r)]
        return vals

    # --- topology
    @staticmethod
    def dims_create(nproc, ndims):
        dims = [1] * ndims
        n, p, factors = nproc, 2, []
        while n > 1:
            while n % p == 0:
                factors.append(p)
                n //= p
            p += 1
        for fct in sorted(factors, reverse=True):
            i = min(range(ndims), key=lambda d: dims[d])
            dims[i] *= fct
        return sorted(dims, reverse=True)

    def cart_create(self, dims):
        self.w.dims = list(dims)
        return 1

    def coords_of(self, rank):
        dims = self.w.dims
        c = []
        for d in reversed(dims):
            c.append(rank % d)
            rank //= d
        return list(reversed(c))

    def rank_of(self, coords):
        r = 0
        for c, d in zip(coords, self.w.dims):
            r = r * d + c
        return r

    def cart_shift(self, direction, disp):
        c = self.coords_of(self.rank)
        d = self.w.dims[direction]
        lo, hi = list(c), list(c)
        lo[direction] -= disp
        hi[direction] += disp
        src = self.rank_of(lo) if 0 <= lo[direction] < d else PROC_NULL
        dst = self.rank_of(hi) if 0 <= hi[direction] < d else PROC_NULL
        return src, dst

    # --- point to point (buffered sends)
    def send(self, arr, off, count, dest, tag):
        if dest == PROC_NULL:
            return
        payload = arr.data[off:off + count]
        assert len(payload) == count, "send past the end of the buffer"
        with self.w.cv:
            self.w.queues[(self.rank, dest, tag)].append(payload)
            self.w.cv.notify_all()

    def recv(self, arr, off, count, source, tag):
        if source == PROC_NULL:
            return
        q = self.w.queues[(source, self.rank, tag)]
        with self.w.cv:
            t0 = time.time()
            while not q:
                if self.w.failed or time.time() - t0 > 600:
                    raise RuntimeError("MPI emulator: receive never satisfied")
                self.w.cv.wait(1.0)
            payload = q.popleft()
        assert len(payload) == count and off + count <= len(arr.data)
        arr.data[off:off + count] = payload

    def sendrecv(self, sarr, soff, scount, dest, stag, rarr, roff, rcount, source, rtag):
        self.send(sarr, soff, scount, dest, stag)
        self.recv(rarr, roff, rcount, source, rtag)

    # --- collectives
    def bcast(self, arr, off, count, root):
        vals = self._exchange(arr.data[off:off + count] if self.rank == root else None)
        arr.data[off:off + count] = vals[root]

    def bcast_scalar(self, value, root):
        return self._exchange(value if self.rank == root else None)[root]

    def scatterv(self, sarr, soff, counts, displs, rarr, roff, rcount, root):
        vals = self._exchange(list(sarr.data) if self.rank == root else None)
        src = vals[root]
        d = displs.data[self.rank]
        rarr.data[roff:roff + rcount] = src[soff + d: soff + d + rcount]

    def gatherv(self, sarr, soff, scount, rarr, roff, counts, displs, root):
        vals = self._exchange(sarr.data[soff:soff + scount])
        if self.rank == root:
            for r in range(self.size):
                d = displs.data[r]
                rarr.data[roff + d: roff + d + counts.data[r]] = vals[r]

    def allgather_scalar(self, value, rarr):
        vals = self._exchange(value)
        rarr.data[0:self.size] = vals

    def allreduce_sum(self, value):
        vals = self._exchange(value)
        acc = vals[0]
        for v in vals[1:]:
            acc = acc + v
        return acc


def fmod(a, b):
    return a - int(a / b) * b if isinstance(a, int) and isinstance(b, int) else math.fmod(a, b)


def idiv(a, b):
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


# ---------------------------------------------------------------------------
# source handling
# ---------------------------------------------------------------------------


def logical_lines(text):
    """Comments stripped, continuations joined, lower-cased."""
    out, buf = [], ""
    for raw in text.splitlines():
        line, inq = [], None
        for ch in raw:
            if inq:
                line.append(ch)
                if ch == inq:
                    inq = None
            elif ch in "'\"":
                inq = ch
                line.append(ch)
            elif ch == "!":
                break
            else:
                line.append(ch)
        s = "".join(line).rstrip()
        if buf:
            s = s.lstrip()
            if s.startswith("&"):
                s = s[1:]
        if s.endswith("&"):
            buf += s[:-1]
            continue
        s = buf + s
        buf = ""
        if s.strip():
            out.append(_lower_outside_quotes(s.strip()))
    return out


def _lower_outside_quotes(s):
    out, inq = [], None
    for ch in s:
        if inq:
            out.append(ch)
            if ch == inq:
                inq = None
        elif ch in "'\"":
            inq = ch
            out.append(ch)
        else:
            out.append(ch.lower())
    return "".join(out)


TOKEN = re.compile(r"""
    (?P<num>(\d+\.\d*|\.\d+|\d+)([ed][+-]?\d+)?(_\d+)?)
  | (?P<dot>\.(and|or|not|eq|ne|lt|le|gt|ge|true|false)\.)
  | (?P<id>[a-z_][a-z0-9_]*)
  | (?P<op>\*\*|//|==|/=|<=|>=|\(/|/\)|[-+*/(),:<>=%])
  | (?P<ws>\s+)
""", re.X)


def tokenize(s):
    toks, pos = [], 0
    while pos < len(s):
        m = TOKEN.match(s, pos)
        if not m:
            raise SyntaxError(f"cannot tokenize at {s[pos:]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        toks.append((kind, m.group(kind)))
    return toks


# AST nodes are tuples: ("num", text) ("name", id) ("call", id, [args]) ("slice", lo, hi)
# ("bin", op, a, b) ("un", op, a) ("cons", [items]) ("logic", value)
class Parser:
    PREC = {".or.": 1, ".and.": 2, ".eqv.": 0, "==": 4, "/=": 4, "<": 4, "<=": 4, ">": 4, ">=": 4,
            ".eq.": 4, ".ne.": 4, ".lt.": 4, ".le.": 4, ".gt.": 4, ".ge.": 4,
            "+": 5, "-": 5, "*": 6, "/": 6, "**": 8}

    def __init__(self, toks):
        self.t, self.i = toks, 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise SyntaxError(f"expected {val}, got {tok}")
        self.i += 1
        return tok

    def expr(self, minp=0):
        kind, val = self.peek()
        if val in ("-", "+"):
            self.take()
            a = self.expr(5 + 1)  # unary +- bind like binary +- (operand may hold * / **)
            left = ("un", val, a)
        elif val == ".not.":
            self.take()
            left = ("un", ".not.", self.expr(3))
        else:
            left = self.atom()
        while True:
            kind, val = self.peek()
            if val not in self.PREC:
                break
            p = self.PREC[val]
            if p < minp:
                break
            self.take()
            right = self.expr(p if val == "**" else p + 1)
            left = ("bin", val, left, right)
        return left

    def atom(self):
        kind, val = self.take()
        if kind == "num":
            return ("num", val)
        if kind == "dot" and val in (".true.", ".false."):
            return ("logic", val == ".true.")
        if val == "(/":
            items = []
            while self.peek()[1] != "/)":
                items.append(self.expr())
                if self.peek()[1] == ",":
                    self.take()
            self.take("/)")
            return ("cons", items)
        if val == "(":
            e = self.expr()
            self.take(")")
            return e
        if kind == "id":
            if self.peek()[1] == "(":
                self.take("(")
                args = []
                while self.peek()[1] != ")":
                    args.append(self.arg())
                    if self.peek()[1] == ",":
                        self.take()
                self.take(")")
                return ("call", val, args)
            return ("name", val)
        raise SyntaxError(f"unexpected token {val!r}")

    def arg(self):
        if self.peek()[1] == ":":
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.expr()
            return ("slice", None, hi)
        e = self.expr()
        if self.peek()[1] == ":":
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.expr()
            return ("slice", e, hi)
        return e


def parse_expr(s):
    p = Parser(tokenize(s))
    e = p.expr()
    if p.i != len(p.t):
        raise SyntaxError(f"trailing tokens in {s!r}: {p.t[p.i:]}")
    return e


# ---------------------------------------------------------------------------
# translation
# ---------------------------------------------------------------------------
MPI_CONST = {"mpi_comm_world": "1", "mpi_real8": "1", "mpi_integer": "2", "mpi_sum": "1",
             "mpi_proc_null": str(PROC_NULL), "mpi_status_size": "6"}
INTRINSIC_REAL = {"dble", "sqrt", "dsqrt", "erf", "real"}


class Sym:
    def __init__(self, typ, dims=None, param=False, alloc=False, init=None):
        self.typ, self.dims, self.param, self.alloc, self.init = typ, dims, param, alloc, init


def split_top(s, sep=","):
    parts, depth, cur, inq = [], 0, "", None
    for ch in s:
        if inq:
            cur += ch
            if ch == inq:
                inq = None
            continue
        if ch in "'\"":
            inq = ch
        elif ch in "(":
            depth += 1
        elif ch in ")":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return [p.strip() for p in parts if p.strip()]


DECL = re.compile(r"^(integer|real|logical|character)\s*(\([^)]*\))?\s*(,[^:]*)?::\s*(.*)$")
DECL_OLD = re.compile(r"^(integer|real|logical)\s*(\([^)]*\))?\s+([a-z].*)$")


class Unit:
    def __init__(self, kind, name, args, result=None):
        self.kind, self.name, self.args, self.result = kind, name, args, result
        self.body, self.syms = [], {}


class Translator:
    def __init__(self, src, overrides=None, check_every=None, with_output=False):
        self.with_output = with_output
        self.lines = logical_lines(src)
        if check_every:
            self.lines = [ln.replace("mod(itc,2000)", f"mod(itc,{int(check_every)})") for ln in self.lines]
        self.overrides = {k.lower(): v for k, v in (overrides or {}).items()}
        self.check_every = check_every
        self.module = {}
        self.units = {}
        self.params = {}
        self.data_init = {}
        self._split_units()

    # --- units and declarations
    def _split_units(self):
        cur = None
        for ln in self.lines:
            m = re.match(r"^module\s+(\w+)$", ln)
            if m:
                cur = Unit("module", m.group(1), [])
                continue
            m = re.match(r"^(pure\s+)?function\s+(\w+)\s*\(([^)]*)\)\s*result\s*\((\w+)\)$", ln)
            if m:
                cur = Unit("function", m.group(2), [a.strip() for a in m.group(3).split(",")], m.group(4))
                self.units[cur.name] = cur
                continue
            m = re.match(r"^subroutine\s+(\w+)\s*(\(([^)]*)\))?$", ln)
            if m:
                args = [a.strip() for a in (m.group(3) or "").split(",") if a.strip()]
                cur = Unit("subroutine", m.group(1), args)
                self.units[cur.name] = cur
                continue
            m = re.match(r"^program\s+(\w+)$", ln)
            if m:
                cur = Unit("program", m.group(1), [])
                self.units["__main__"] = cur
                continue
            if re.match(r"^end\s*(module|subroutine|function|program)\b", ln):
                if cur is not None and cur.kind == "module":
                    self.module = cur.syms
                cur = None
                continue
            if cur is None:
                continue
            if ln.startswith("use ") or ln == "implicit none" or ln.startswith("contains"):
                continue
            if self._declaration(cur, ln):
                continue
            cur.body.append(ln)

    def _declaration(self, unit, ln):
        m = DECL.match(ln)
        if m:
            typ, attrs, names = m.group(1), m.group(3) or "", m.group(4)
        else:
            m2 = DECL_OLD.match(ln)
            if not m2 or "=" in ln.split("(")[0]:
                if ln.startswith("data "):
                    self._data(unit, ln)
                    return True
                return False
            typ, attrs, names = m2.group(1), "", m2.group(3)
        if typ == "character":
            for item in split_top(names):
                unit.syms[item.split("=")[0].split("(")[0].strip()] = Sym("character")
            return True
        param = "parameter" in attrs
        alloc = "allocatable" in attrs
        for item in split_top(names):
            init = None
            if "=" in item and not item.startswith("("):
                item, init = item.split("=", 1)
                item, init = item.strip(), init.strip()
            mm = re.match(r"^(\w+)\s*(\((.*)\))?$", item)
            name, dims = mm.group(1), mm.group(3)
            unit.syms[name] = Sym("int" if typ == "integer" else ("logical" if typ == "logical" else "real"),
                                  dims=split_top(dims) if dims else None, param=param, alloc=alloc, init=init)
        return True

    def _data(self, unit, ln):
        for m in re.finditer(r"(\w+)\s*/([^/]*)/", ln[5:]):
            name, vals = m.group(1), m.group(2)
            items = []
            for v in split_top(vals):
                if "*" in v:
                    n, val = v.split("*")
                    items += [val.strip()] * int(n)
                else:
                    items.append(v)
            unit.syms[name].init = ("data", items)

    # --- expression codegen
    def sym(self, unit, name):
        if name in unit.syms:
            return unit.syms[name], False
        if name in self.module:
            return self.module[name], True
        return None, False

    def ref(self, unit, name):
        if name in MPI_CONST:
            return MPI_CONST[name]
        s, glob = self.sym(unit, name)
        if s is None:
            raise NameError(f"{unit.name}: unknown name {name}")
        if unit.kind == "function" and name == unit.name:
            return f"v_{unit.result}"
        return f"S.{name}" if glob else f"v_{name}"

    def typeof(self, unit, e):
        k = e[0]
        if k == "num":
            return "real" if re.search(r"[.ed]", e[1]) else "int"
        if k == "logic":
            return "logical"
        if k == "name":
            if e[1] in MPI_CONST:
                return "int"
            s, _ = self.sym(unit, e[1])
            return s.typ
        if k == "call":
            n = e[1]
            if n in INTRINSIC_REAL:
                return "real"
            if n in ("int",):
                return "int"
            if n in ("mod", "abs", "min", "max"):
                ts = [self.typeof(unit, a) for a in e[2]]
                return "real" if "real" in ts else "int"
            if n in self.units:
                return "real"
            s, _ = self.sym(unit, n)
            return s.typ
        if k == "bin":
            if e[1] in Parser.PREC and Parser.PREC[e[1]] <= 4:
                return "logical"
            ta, tb = self.typeof(unit, e[2]), self.typeof(unit, e[3])
            return "real" if "real" in (ta, tb) else "int"
        if k == "un":
            return "logical" if e[1] == ".not." else self.typeof(unit, e[2])
        raise TypeError(e)

    def num(self, text):
        t = text.split("_")[0]
        if re.search(r"[.ed]", t):
            if "d" in t:
                return repr(float(t.replace("d", "e")))
            return repr(f32(float(t)))
        return str(int(t))

    def ex(self, unit, e, elem=None):
        """Python for expression e; elem maps whole-array names to a flat index."""
        k = e[0]
        if k == "num":
            return self.num(e[1])
        if k == "logic":
            return "True" if e[1] else "False"
        if k == "name":
            n = e[1]
            s, _ = self.sym(unit, n)
            if s is not None and s.dims is not None and elem is not None:
                return f"{self.ref(unit, n)}.data[{elem}]"
            if s is not None and s.param and n in self.params:
                return repr(self.params[n])
            return self.ref(unit, n)
        if k == "un":
            a = self.ex(unit, e[2], elem)
            return f"(not {a})" if e[1] == ".not." else f"({e[1]}{a})"
        if k == "bin":
            op = e[1]
            a, b = self.ex(unit, e[2], elem), self.ex(unit, e[3], elem)
            if op == "**":
                base = e[3]
                if base[0] == "num" and float(base[1].replace("d", "e")) in (2.0, 3.0):
                    n = int(float(base[1].replace("d", "e")))
                    return f"({a}*{a})" if n == 2 else f"(({a}*{a})*{a})"
                return f"({a}**{b})"
            if op == "/" and self.typeof(unit, e[2]) == "int" and self.typeof(unit, e[3]) == "int":
                return f"idiv({a}, {b})"
            pyop = {".and.": "and", ".or.": "or", "==": "==", "/=": "!=", ".eq.": "==", ".ne.": "!=",
                    ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">="}.get(op, op)
            return f"({a} {pyop} {b})"
        if k == "call":
            n, args = e[1], e[2]
            if n in ("dble", "real") and n not in unit.syms:
                inner = self.ex(unit, args[0], elem)
                return f"float({inner})" if n == "dble" else f"f32(float({inner}))"
            if n in ("sqrt", "dsqrt"):
                return f"math.sqrt({self.ex(unit, args[0], elem)})"
            if n == "erf":
                return f"math.erf({self.ex(unit, args[0], elem)})"
            if n == "mod":
                return f"fmod({self.ex(unit, args[0], elem)}, {self.ex(unit, args[1], elem)})"
            if n in ("abs", "min", "max", "int"):
                return f"{n}({', '.join(self.ex(unit, a, elem) for a in args)})"
            if n == "mpi_wtime":
                return "mpi.wtime()"
            if n in self.units and self.units[n].kind == "function":
                return f"fn_{n}({', '.join(self.ex(unit, a, elem) for a in args)})"
            # array element
            idx = ", ".join(self.ex(unit, a, elem) for a in args)
            return f"{self.ref(unit, n)}[{idx}]" if len(args) > 1 else f"{self.ref(unit, n)}[{idx}]"
        if k == "cons":
            return "[" + ", ".join(self.ex(unit, a, elem) for a in e[1]) + "]"
        raise TypeError(e)

    # --- buffers for MPI calls: (array expr, flat offset expr) or scalar
    def buf(self, unit, e):
        if e[0] == "name":
            s, _ = self.sym(unit, e[1])
            if s.dims is not None:
                return ("arr", self.ref(unit, e[1]), "0")
            return ("scalar", self.ref(unit, e[1]), None)
        if e[0] == "call":
            a = self.ref(unit, e[1])
            idx = ", ".join(self.ex(unit, x) for x in e[2])
            return ("arr", a, f"{a}.off(({idx},))")
        raise TypeError(e)

    def mpi_call(self, unit, name, args):
        A = [parse_expr(a) for a in args]
        E = lambda i: self.ex(unit, A[i])  # noqa: E731
        if name in ("mpi_init", "mpi_finalize"):
            return ["pass"]
        if name == "mpi_comm_size":
            return [f"{self.ref(unit, A[1][1])} = mpi.size"]
        if name == "mpi_comm_rank":
            return [f"{self.ref(unit, A[1][1])} = mpi.rank"]
        if name == "mpi_barrier":
            return ["mpi.barrier()"]
        if name == "mpi_dims_create":
            d = self.ref(unit, A[2][1])
            return [f"_dc = mpi.dims_create({E(0)}, {E(1)})", f"for _t in range({E(1)}): {d}.data[_t] = _dc[_t]"]
        if name == "mpi_cart_create":
            d = self.ref(unit, A[2][1])
            return [f"{self.ref(unit, A[5][1])} = mpi.cart_create({d}.data[0:{E(1)}])"]
        if name == "mpi_cart_coords":
            c = self.ref(unit, A[3][1])
            return [f"_cc = mpi.coords_of({E(1)})", f"for _t in range({E(2)}): {c}.data[_t] = _cc[_t]"]
        if name == "mpi_cart_shift":
            return [f"{self.ref(unit, A[3][1])}, {self.ref(unit, A[4][1])} = mpi.cart_shift({E(1)}, {E(2)})"]
        if name == "mpi_bcast":
            b = self.buf(unit, A[0])
            if b[0] == "scalar":
                return [f"{b[1]} = mpi.bcast_scalar({b[1]}, {E(3)})"]
            return [f"mpi.bcast({b[1]}, {b[2]}, {E(1)}, {E(3)})"]
        if name == "mpi_scatterv":
            s, r = self.buf(unit, A[0]), self.buf(unit, A[4])
            return [f"mpi.scatterv({s[1]}, {s[2]}, {E(1)}, {E(2)}, {r[1]}, {r[2]}, {E(5)}, {E(7)})"]
        if name == "mpi_gatherv":
            s = self.buf(unit, A[0])
            r = self.buf(unit, A[3])
            return [f"mpi.gatherv({s[1]}, {s[2]}, {E(1)}, {r[1]}, ({r[2]}) if mpi.rank == {E(7)} else 0, "
                    f"{E(4)}, {E(5)}, {E(7)})"]
        if name == "mpi_allgather":
            return [f"mpi.allgather_scalar({E(0)}, {self.ref(unit, A[3][1])})"]
        if name == "mpi_allreduce":
            return [f"{self.ref(unit, A[1][1])} = mpi.allreduce_sum({E(0)})"]
        if name == "mpi_sendrecv":
            s, r = self.buf(unit, A[0]), self.buf(unit, A[5])
            return [f"mpi.sendrecv({s[1]}, {s[2]}, {E(1)}, {E(3)}, {E(4)}, {r[1]}, {r[2]}, {E(6)}, {E(8)}, {E(9)})"]
        if name == "mpi_send":
            s = self.buf(unit, A[0])
            return [f"mpi.send({s[1]}, {s[2]}, {E(1)}, {E(3)}, {E(4)})"]
        if name == "mpi_recv":
            r = self.buf(unit, A[0])
            return [f"mpi.recv({r[1]}, {r[2]}, {E(1)}, {E(3)}, {E(4)})"]
        raise NotImplementedError(name)

    # --- formatted output to numbered units (with_output)
    def io_stmt(self, unit, ln):
        """Python for an open / write / close on a numbered unit, None for
        anything else (stdout, internal files, other statements)."""
        m = re.match(r"^open\s*\((.*)\)$", ln)
        if m:
            mm = re.search(r"unit\s*=\s*(\d+)", m.group(1))
            return f"fio_open(S, {int(mm.group(1))})" if mm else None
        if re.match(r"^close\s*\(\s*\d+\s*\)$", ln) or re.match(r"^\d+\s+format", ln):
            return "pass"
        m = re.match(r"^write\s*\(\s*(\d+)\s*,\s*(\*|\d+)\s*\)\s*(.*)$", ln)
        if not m:
            return None
        u, fmt, items = int(m.group(1)), m.group(2), split_top(m.group(3))
        vals = []
        for it in items:
            if it[0] in "'\"":
                vals.append(repr(it[1:-1]))
            else:
                vals.append(self.ex(unit, parse_expr(it)))
        if fmt == "*":
            return f"fio_write_list(S, {u}, [{', '.join(vals)}])"
        text = unit.fmts[fmt]
        return f"fio_write_fmt(S, {u}, {text!r}, [{', '.join(vals)}])"

    # --- array allocation code
    def bounds(self, unit, dims):
        out = []
        for d in dims:
            if ":" in d:
                lo, hi = d.split(":", 1)
                out.append(f"({self.ex(unit, parse_expr(lo))}, {self.ex(unit, parse_expr(hi))})")
            else:
                out.append(f"(1, {self.ex(unit, parse_expr(d))})")
        return "[" + ", ".join(out) + "]"

    # --- statements
    def stmt(self, unit, ln, out, ind):
        P = " " * ind

        def emit(s):
            out.append(P + s)

        if self.with_output:
            io = self.io_stmt(unit, ln)
            if io is not None:
                emit(io)
                return
        if re.match(r"^(write|open|close|print|deallocate)\b", ln) or re.match(r"^\d+\s+format", ln):
            emit("pass")
            return
        if ln == "return":
            emit("return" + (f" v_{unit.result}" if unit.kind == "function" else ""))
            return
        if ln == "stop":
            emit("raise Stop()")
            return
        m = re.match(r"^allocate\s*\((.*)\)$", ln)
        if m:
            for item in split_top(m.group(1)):
                mm = re.match(r"^(\w+)\s*\((.*)\)$", item)
                name, dims = mm.group(1), split_top(mm.group(2))
                s, _ = self.sym(unit, name)
                emit(f"{self.ref(unit, name)} = FArray({self.bounds(unit, dims)}, '{s.typ}')")
            return
        m = re.match(r"^call\s+(\w+)\s*(\((.*)\))?$", ln)
        if m:
            name, args = m.group(1), split_top(m.group(3) or "")
            if name.startswith("mpi_"):
                for s in self.mpi_call(unit, name, args):
                    emit(s)
                return
            if name == "output_ascii" and not self.with_output:
                emit("pass")
                return
            call = f"sub_{name}(S, mpi{''.join(', ' + self.ex(unit, parse_expr(a)) for a in args)})"
            emit(call)
            if name == "check":
                emit("S._checks.append((S.itc, S.erroru, S.errort))")
            return
        # assignment
        m = re.match(r"^([a-z_][\w]*\s*(\([^=]*\))?)\s*=\s*(.*)$", ln)
        if m and not ln.startswith("if"):
            lhs, rhs = m.group(1).strip(), m.group(3)
            L = parse_expr(lhs)
            name = L[1]
            s, _ = self.sym(unit, name)
            if s is not None and s.typ == "character":
                emit("pass")
                return
            R = parse_expr(rhs)
            if L[0] == "name" and s is not None and s.dims is not None:
                # whole-array assignment, elementwise over the flat storage
                a = self.ref(unit, name)
                emit(f"for _n in range(len({a}.data)):")
                emit(f"    {a}.data[_n] = {self.ex(unit, R, elem='_n')}")
                return
            if L[0] == "call" and any(x[0] == "slice" for x in L[2]):
                self.section_assign(unit, L, R, emit)
                return
            emit(f"{self.ex(unit, L)} = {self.ex(unit, R)}")
            return
        raise SyntaxError(f"{unit.name}: unhandled statement {ln!r}")

    def section_assign(self, unit, L, R, emit):
        """a(lo:hi) = expr-of-sections, or a(i,:) = (/.../)."""
        a = self.ref(unit, L[1])
        sl = [i for i, x in enumerate(L[2]) if x[0] == "slice"]
        assert len(sl) == 1, "only one sectioned dimension is supported"
        d = sl[0]
        lo = L[2][d][1]
        hi = L[2][d][2]
        lo_s = self.ex(unit, lo) if lo is not None else f"{a}.lb[{d}]"
        hi_s = self.ex(unit, hi) if hi is not None else f"{a}.lb[{d}] + {a}.ext[{d}] - 1"
        idx = lambda t: ", ".join("(" + lo_s + " + " + t + ")" if i == d else self.ex(unit, x)  # noqa: E731
                                  for i, x in enumerate(L[2]))
        if R[0] == "cons":
            emit(f"_rhs = {self.ex(unit, R)}")
        else:
            # every section in R is 1-D with an explicit lower bound; index it by _t
            def sec(e):
                if e[0] == "call" and any(x[0] == "slice" for x in e[2]):
                    args = []
                    for x in e[2]:
                        if x[0] == "slice":
                            args.append(f"({self.ex(unit, x[1])} + _t)")
                        else:
                            args.append(self.ex(unit, x))
                    return f"{self.ref(unit, e[1])}[{', '.join(args)}]"
                if e[0] == "bin":
                    return f"({sec(e[2])} {e[1]} {sec(e[3])})"
                if e[0] == "un":
                    return f"({e[1]}{sec(e[2])})"
                return self.ex(unit, e)
            emit(f"_rhs = [{sec(R)} for _t in range(({hi_s}) - ({lo_s}) + 1)]")
        emit(f"for _t in range(({hi_s}) - ({lo_s}) + 1):")
        emit(f"    {a}[{idx('_t')}] = _rhs[_t]")

    def block(self, unit, body, out, ind):
        """Translate a statement list with do / if nesting."""
        i = 0
        stack = []
        P = lambda n: " " * n  # noqa: E731
        cur = ind
        for ln in body:
            m = re.match(r"^do\s+while\s*\((.*)\)$", ln)
            if m:
                out.append(P(cur) + f"while {self.ex(unit, parse_expr(m.group(1)))}:")
                stack.append("do")
                cur += 4
                continue
            m = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", ln)
            if m:
                v = self.ref(unit, m.group(1))
                parts = split_top(m.group(2))
                lo, hi = self.ex(unit, parse_expr(parts[0])), self.ex(unit, parse_expr(parts[1]))
                step = self.ex(unit, parse_expr(parts[2])) if len(parts) > 2 else "1"
                if step == "1":
                    out.append(P(cur) + f"for {v} in range({lo}, ({hi}) + 1):")
                else:
                    out.append(P(cur) + f"for {v} in range({lo}, ({hi}) + ({step}), {step}):")
                stack.append("do")
                cur += 4
                continue
            if re.match(r"^end\s*do$", ln):
                assert stack.pop() == "do"
                out.append(P(cur) + "pass")
                cur -= 4
                continue
            m = re.match(r"^if\s*\((.*)\)\s*then$", ln)
            if m:
                out.append(P(cur) + f"if {self.ex(unit, parse_expr(m.group(1)))}:")
                stack.append("if")
                cur += 4
                continue
            m = re.match(r"^else\s*if\s*\((.*)\)\s*then$", ln)
            if m:
                out.append(P(cur) + "pass")
                out.append(P(cur - 4) + f"elif {self.ex(unit, parse_expr(m.group(1)))}:")
                continue
            if ln == "else":
                out.append(P(cur) + "pass")
                out.append(P(cur - 4) + "else:")
                continue
            if re.match(r"^end\s*if$", ln):
                assert stack.pop() == "if"
                out.append(P(cur) + "pass")
                cur -= 4
                continue
            m = re.match(r"^if\s*\((.*)\)\s*(\w.*)$", ln)
            if m:
                # single-line if: find the matching parenthesis of the condition
                depth, k = 0, ln.index("(")
                for k2 in range(k, len(ln)):
                    depth += ln[k2] == "("
                    depth -= ln[k2] == ")"
                    if depth == 0:
                        break
                cond, rest = ln[k + 1:k2], ln[k2 + 1:].strip()
                out.append(P(cur) + f"if {self.ex(unit, parse_expr(cond))}:")
                self.stmt(unit, rest, out, cur + 4)
                continue
            self.stmt(unit, ln, out, cur)
        assert not stack, f"{unit.name}: unbalanced blocks"

    # --- whole program
    def module_init(self, out):
        out.append("def init_module(S):")
        for name, s in self.module.items():
            if s.param:
                if name in self.overrides:
                    val = self.overrides[name]
                else:
                    val = eval(self.ex(Unit("module", "commondata", []), parse_expr(s.init)),  # noqa: S307
                               {"idiv": idiv, "f32": f32, "math": math, "S": None})
                if s.typ == "real":
                    val = float(val)
                self.params[name] = val
                out.append(f"    S.{name} = {val!r}")
        for name, s in self.module.items():
            if s.param:
                continue
            if s.dims is not None and not s.alloc:
                dims = self.bounds(Unit("module", "commondata", []), s.dims)
                out.append(f"    S.{name} = FArray({dims}, '{s.typ}')")
                if isinstance(s.init, tuple):
                    vals = ", ".join(self.ex(Unit("module", "c", []), parse_expr(v)) for v in s.init[1])
                    out.append(f"    S.{name}.data[:] = [{vals}]")
            elif s.dims is not None:
                out.append(f"    S.{name} = None")
            elif s.typ == "character":
                continue
            else:
                init = self.ex(Unit("module", "c", []), parse_expr(s.init)) if s.init else (
                    "0.0" if s.typ == "real" else ("False" if s.typ == "logical" else "0"))
                out.append(f"    S.{name} = {init}")
        out.append("    S._checks = []")

    def unit_code(self, unit, out):
        unit.fmts = {}
        for ln in unit.body:
            m = re.match(r"^(\d+)\s+format\s*(\(.*\))$", ln)
            if m:
                unit.fmts[m.group(1)] = m.group(2)
        if unit.kind == "function":
            args = ", ".join(f"v_{a}" for a in unit.args)
            out.append(f"def fn_{unit.name}({args}):")
        elif unit.kind == "subroutine":
            args = "".join(f", v_{a}" for a in unit.args)
            out.append(f"def sub_{unit.name}(S, mpi{args}):")
        else:
            out.append("def main(S, mpi):")
        for name, s in unit.syms.items():
            if name in unit.args or s.typ == "character":
                continue
            if unit.kind == "function" and name == unit.name:
                continue
            if s.dims is not None and not s.alloc and not all(d == ":" for d in s.dims):
                out.append(f"    v_{name} = FArray({self.bounds(unit, s.dims)}, '{s.typ}')")
            elif s.dims is None:
                out.append(f"    v_{name} = {'0.0' if s.typ == 'real' else ('False' if s.typ == 'logical' else '0')}")
            else:
                out.append(f"    v_{name} = None")
        if unit.kind == "function":
            out.append(f"    v_{unit.result} = 0.0")
        self.block(unit, unit.body, out, 4)
        if unit.kind == "function":
            out.append(f"    return v_{unit.result}")
        out.append("")

    def python(self):
        out = []
        self.module_init(out)
        out.append("")
        for name, u in self.units.items():
            self.unit_code(u, out)
        return "\n".join(out) + "\n"


def run(src, nranks, overrides=None, check_every=None, with_output=False):
    """Translate and run a reference program on nranks emulated ranks.
    Returns the per-rank module states after the program ends (with_output:
    each state's _io maps a unit number to the text written to it)."""
    import f90fmt
    tr = Translator(src, overrides, check_every, with_output)
    code = tr.python()
    ns = {"math": math, "FArray": FArray, "Stop": Stop, "fmod": fmod, "idiv": idiv, "f32": f32,
          "fio_open": f90fmt.fio_open, "fio_write_list": f90fmt.fio_write_list,
          "fio_write_fmt": f90fmt.fio_write_fmt}
    exec(compile(code, "<reference-translation>", "exec"), ns)  # noqa: S102
    world = World(nranks)
    states = [type("State", (), {})() for _ in range(nranks)]
    errors = []

    def rank_main(r):
        S = states[r]
        ns["init_module"](S)
        try:
            ns["main"](S, Comm(world, r))
        except Stop:
            pass
        except BaseException as e:  # noqa: BLE001
            errors.append((r, e))
            world.failed = True
            world.barrier.abort()

    threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(nranks)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise RuntimeError(f"rank {errors[0][0]} failed") from errors[0][1]
    return states, code
