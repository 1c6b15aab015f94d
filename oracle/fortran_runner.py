"""Run the reference's own Fortran routines on the host, without a compiler.

TEST INFRASTRUCTURE ONLY.  Neither the library nor the bench imports this
module.  It exists because neither this container nor the GPU machine has a
Fortran compiler or MPI, so the reference (derek-teaney/lceqcd, fixed-form
Fortran 77/90 + MPI, built by ``obj/Makefile`` with gfortran
``-ffixed-line-length-256``) cannot be built; instead its unmodified source
files are parsed and executed statement by statement.

Only the language subset the Monte Carlo path uses is implemented:

* fixed-form source (label columns 1-5, continuation in column 6, ``c``/``C``/
  ``*``/``!`` comment lines, ``!`` trailing comments), ``INCLUDE`` files;
* ``SUBROUTINE``/``PROGRAM`` units, ``IMPLICIT``, type declarations,
  ``DIMENSION``, ``PARAMETER``, ``COMMON``, automatic arrays, explicit lower
  bounds (``even:odd``), assumed-size dummies;
* ``DO`` (block and labelled, shared terminators), block and logical ``IF``,
  ``WHERE``/``ELSEWHERE``, ``GOTO``, ``CALL``, ``RETURN``, ``STOP``,
  ``CONTINUE``, assignments to scalars, elements, sections and whole arrays;
* argument passing by reference with sequence association (an array element
  passed to an array dummy starts the dummy's storage there, as the
  ``multall*`` calls rely on);
* the intrinsics the path calls (``sqrt exp log cos sin acos abs aint int nint
  real float dble cmplx conjg aimag mod min max sum count dot_product sign``),
  with whole-array arithmetic;
* MPI reduced to one rank (reductions and gathers copy their send buffer,
  topology calls return rank 0 and coordinate 0), list-directed ``READ`` of
  the input file, ``WRITE`` to a file unit captured as a list of values, and
  every other ``WRITE``/``OPEN``/``CLOSE``/``FORMAT`` ignored.

``call random_number(x)`` draws from a uniform stream the caller supplies, in
the order the reference consumes it.

Arithmetic: ``real_kind=4`` keeps the reference's default REAL (float32, and
complex64 for COMPLEX); ``real_kind=8`` promotes default REAL and COMPLEX to
64 bits, as gfortran's ``-fdefault-real-8`` would, which is how the FP64
restatement in ``lce_oracle.c`` is pinned.  Integer division and ``mod``
truncate toward zero; ``x**2`` is ``x*x``; ``sum``/``dot_product`` accumulate
sequentially; locals start as NaN (REAL/COMPLEX) so that a read before a
write shows up in the results.
"""
from __future__ import annotations

import os
import re
import warnings

import numpy as np

# ----------------------------------------------------------------------------
# source handling


class FortranError(RuntimeError):
    pass


def _strip_comment(text: str) -> str:
    """Drop a trailing '!' comment that is not inside a string."""
    q = None
    for i, ch in enumerate(text):
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "!":
            return text[:i]
    return text


def _lower_outside_strings(text: str) -> str:
    out = []
    q = None
    for ch in text:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        else:
            out.append(ch.lower())
    return "".join(out)


def read_fixed_form(path: str, include_dirs: list[str]) -> list[tuple]:
    """Logical statements of a fixed-form file: (label, text, origin)."""
    with open(path, encoding="latin-1") as fh:
        raw = fh.read().split("\n")
    stmts = []
    for n, line in enumerate(raw, 1):
        line = line.rstrip("\r")
        if not line.strip():
            continue
        if line[0] in "cC*!":
            continue
        if "\t" in line[:6]:
            head, _, tail = line.partition("\t")
            line = head.ljust(6) + tail
        label_field = line[:5]
        cont = len(line) > 5 and line[5] not in " 0"
        body = _strip_comment(line[6:])
        if cont:
            if not stmts:
                raise FortranError(f"{path}:{n}: continuation without a statement")
            lab, txt, org = stmts[-1]
            stmts[-1] = (lab, txt + body, org)
            continue
        if not body.strip() and not label_field.strip():
            continue
        lab = label_field.strip()
        stmts.append((int(lab) if lab else None, body, f"{os.path.basename(path)}:{n}"))
    out = []
    for lab, txt, org in stmts:
        txt = _lower_outside_strings(txt).strip()
        if not txt:
            if lab is not None:
                out.append((lab, "continue", org))
            continue
        m = re.match(r"include\s*'([^']+)'\s*$", txt)
        if m:
            name = m.group(1)
            if name in ("mpif.h",):
                out.append((lab, "use mpi", org))
                continue
            for d in include_dirs:
                p = os.path.join(d, name)
                if os.path.exists(p):
                    out.extend(read_fixed_form(p, include_dirs))
                    break
            else:
                raise FortranError(f"{org}: include file {name} not found")
            continue
        out.append((lab, txt, org))
    return out


# ----------------------------------------------------------------------------
# expressions

_DOT_OPS = ("eq", "ne", "lt", "le", "gt", "ge", "and", "or", "not", "eqv", "neqv", "true", "false")
_TOKEN_RE = re.compile(r"""
    (?P<ws>\s+)
  | (?P<str>'(?:[^']|'')*'|"(?:[^"]|"")*")
  | (?P<dotop>\.(?:eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv|true|false)\.)
  | (?P<num>(?:\d+\.(?!(?:eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv)\.)\d*|\.\d+|\d+)(?:[ed][+-]?\d+)?)
  | (?P<name>[a-z_][a-z0-9_]*)
  | (?P<op>\*\*|//|==|/=|<=|>=|\(/|/\)|[-+*/()<>,:=%])
""", re.X)


def tokenize(text: str):
    toks = []
    pos = 0
    while pos < len(text):
        m = _TOKEN_RE.match(text, pos)
        if not m:
            raise FortranError(f"cannot tokenize {text[pos:pos + 20]!r} in {text!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        val = m.group(kind)
        if kind == "dotop":
            val = val[1:-1]
            if val in ("true", "false"):
                toks.append(("lit", ("l", val == "true")))
            else:
                toks.append(("op", {"eq": "==", "ne": "/=", "lt": "<", "le": "<=", "gt": ">", "ge": ">="}
                             .get(val, "." + val + ".")))
            continue
        if kind == "num":
            toks.append(("lit", ("n", val)))
        elif kind == "str":
            toks.append(("lit", ("s", val[1:-1].replace(val[0] * 2, val[0]))))
        elif kind == "name":
            toks.append(("name", val))
        else:
            toks.append(("op", val))
    toks.append(("end", None))
    return toks


class _P:
    """Recursive-descent parser for one expression; AST nodes are tuples."""

    def __init__(self, text):
        self.t = tokenize(text)
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k]

    def take(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def expect(self, op):
        tok = self.take()
        if tok != ("op", op):
            raise FortranError(f"expected {op!r}, got {tok}")

    def at(self, op):
        return self.peek() == ("op", op)

    def parse(self):
        e = self.expr()
        if self.peek()[0] != "end":
            raise FortranError(f"trailing tokens {self.t[self.i:]}")
        return e

    def expr(self):
        return self.eqv()

    def eqv(self):
        a = self.or_()
        while self.peek() in (("op", ".eqv."), ("op", ".neqv.")):
            op = self.take()[1]
            a = ("bin", op, a, self.or_())
        return a

    def or_(self):
        a = self.and_()
        while self.at(".or."):
            self.take()
            a = ("bin", ".or.", a, self.and_())
        return a

    def and_(self):
        a = self.not_()
        while self.at(".and."):
            self.take()
            a = ("bin", ".and.", a, self.not_())
        return a

    def not_(self):
        if self.at(".not."):
            self.take()
            return ("not", self.not_())
        return self.rel()

    def rel(self):
        a = self.concat()
        if self.peek()[0] == "op" and self.peek()[1] in ("==", "/=", "<", "<=", ">", ">="):
            op = self.take()[1]
            a = ("bin", op, a, self.concat())
        return a

    def concat(self):
        a = self.add()
        while self.at("//"):
            self.take()
            a = ("bin", "//", a, self.add())
        return a

    def add(self):
        if self.at("-") or self.at("+"):
            op = self.take()[1]
            a = self.mul()
            a = ("neg", a) if op == "-" else a
        else:
            a = self.mul()
        while self.at("+") or self.at("-"):
            op = self.take()[1]
            a = ("bin", op, a, self.mul())
        return a

    def mul(self):
        a = self.power()
        while self.at("*") or self.at("/"):
            op = self.take()[1]
            a = ("bin", op, a, self.power())
        return a

    def power(self):
        a = self.unary()
        if self.at("**"):
            self.take()
            return ("bin", "**", a, self.power_rhs())
        return a

    def power_rhs(self):
        if self.at("-") or self.at("+"):
            op = self.take()[1]
            b = self.power_rhs()
            return ("neg", b) if op == "-" else b
        return self.power()

    def unary(self):
        # gfortran accepts a sign after an operator (a*-b)
        if self.at("-") or self.at("+"):
            op = self.take()[1]
            b = self.power()
            return ("neg", b) if op == "-" else b
        return self.primary()

    def primary(self):
        tok = self.take()
        if tok[0] == "lit":
            return ("lit",) + tok[1]
        if tok == ("op", "("):
            # complex constant (re, im) or parenthesised expression
            e = self.expr()
            if self.at(","):
                self.take()
                e2 = self.expr()
                self.expect(")")
                return ("cmplx_lit", e, e2)
            self.expect(")")
            return ("paren", e)
        if tok == ("op", "(/"):
            items = []
            if not self.at("/)"):
                items.append(self.expr())
                while self.at(","):
                    self.take()
                    items.append(self.expr())
            self.expect("/)")
            return ("arrcons", items)
        if tok[0] == "name":
            name = tok[1]
            if self.at("("):
                self.take()
                args = []
                if not self.at(")"):
                    args.append(self.arg())
                    while self.at(","):
                        self.take()
                        args.append(self.arg())
                self.expect(")")
                return ("ref", name, args)
            return ("name", name)
        raise FortranError(f"unexpected token {tok}")

    def arg(self):
        # section lo:hi[:st], keyword name=expr, or expression
        if self.peek()[0] == "name" and self.peek(1) == ("op", "="):
            kw = self.take()[1]
            self.take()
            return ("kw", kw, self.expr())
        lo = hi = st = None
        if not self.at(":"):
            lo = self.expr()
            if not self.at(":"):
                return lo
        self.take()
        if not (self.at(",") or self.at(")") or self.at(":")):
            hi = self.expr()
        if self.at(":"):
            self.take()
            st = self.expr()
        return ("sec", lo, hi, st)


def parse_expr(text: str):
    return _P(text).parse()


def split_top(text: str, sep: str = ",") -> list[str]:
    """Split at top-level separators (outside parentheses and strings)."""
    out, depth, q, cur = [], 0, None, []
    for ch in text:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
            continue
        cur.append(ch)
    out.append("".join(cur))
    return [s.strip() for s in out]


def match_paren(text: str, start: int) -> int:
    """Index of the ')' matching the '(' at text[start]."""
    depth, q = 0, None
    for i in range(start, len(text)):
        ch = text[i]
        if q:
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                return i
    raise FortranError(f"unbalanced parentheses in {text!r}")


# ----------------------------------------------------------------------------
# runtime values


class Ref:
    """A scalar storage location: element ``idx`` of a 1-D numpy buffer."""
    __slots__ = ("buf", "idx")

    def __init__(self, buf, idx):
        self.buf = buf
        self.idx = idx

    def get(self):
        return self.buf[self.idx]

    def set(self, v):
        self.buf[self.idx] = v


class CharVar:
    __slots__ = ("value", "length")

    def __init__(self, length):
        self.value = ""
        self.length = length

    def get(self):
        return self.value

    def set(self, v):
        self.value = str(v)[: self.length] if self.length else str(v)


class Arr:
    """A Fortran array over a 1-D buffer: column-major, any lower bounds."""
    __slots__ = ("buf", "off", "lo", "ext", "strides", "size", "assumed")

    def __init__(self, buf, off, lo, ext, assumed=False, dummy=False):
        self.buf, self.off, self.lo, self.ext = buf, off, list(lo), list(ext)
        self.assumed = assumed
        st, s = [], 1
        for e in self.ext:
            st.append(s)
            s *= e
        self.strides, self.size = st, s
        # a dummy may be declared larger than the actual's storage (the
        # multall* HELP(2, MAXSIZE) dummies get automatic arrays of ownhalfvol
        # sites); only accesses beyond the storage are errors
        if off + s > len(buf) and not assumed and not dummy:
            raise FortranError(f"array of {s} elements at offset {off} exceeds its storage ({len(buf)})")

    def index(self, subs):
        if len(subs) != len(self.ext):
            raise FortranError(f"rank mismatch: {len(subs)} subscripts for rank {len(self.ext)}")
        k = self.off
        last = len(subs) - 1
        for d, (i, lo, e, st) in enumerate(zip(subs, self.lo, self.ext, self.strides)):
            r = int(i) - lo
            if r < 0 or (r >= e and not (self.assumed and d == last)):
                raise FortranError(f"subscript {int(i)} out of bounds [{lo}, {lo + e - 1}] in dimension {d + 1}")
            k += r * st
        if k >= len(self.buf):
            raise FortranError("element beyond the array's storage")
        return k

    def view(self):
        n = self.size
        if self.off + n > len(self.buf):
            raise FortranError("whole-array use of an assumed-size array beyond its storage")
        return self.buf[self.off:self.off + n].reshape(self.ext, order="F")


# ----------------------------------------------------------------------------
# types and arithmetic


class Kinds:
    def __init__(self, real_kind: int):
        self.real = np.float64 if real_kind == 8 else np.float32
        self.cplx = np.complex128 if real_kind == 8 else np.complex64
        self.int = np.int64


def _cat(x):
    if isinstance(x, (bool, np.bool_)):
        return "l"
    if isinstance(x, (int, np.integer)):
        return "i"
    if isinstance(x, str):
        return "s"
    if isinstance(x, np.ndarray):
        k = x.dtype.kind
        return {"b": "l", "i": "i", "u": "i", "f": "r", "c": "c", "U": "s", "O": "s"}[k]
    if isinstance(x, (np.floating, float)):
        return "r"
    if isinstance(x, (np.complexfloating, complex)):
        return "c"
    raise FortranError(f"value of unsupported type {type(x)}")


def _bits(x):
    dt = x.dtype if isinstance(x, (np.ndarray, np.generic)) else np.dtype(type(x))
    if dt.kind == "c":
        return dt.itemsize * 4
    return dt.itemsize * 8


def _result_dtype(a, b):
    ca, cb = _cat(a), _cat(b)
    if ca == "i" and cb == "i":
        return None
    bits = max(_bits(x) for x, c in ((a, ca), (b, cb)) if c in "rc")
    if "c" in (ca, cb):
        return np.complex128 if bits > 32 else np.complex64
    return np.float64 if bits > 32 else np.float32


def _conv(x, dt):
    if isinstance(x, np.ndarray):
        return x.astype(dt, copy=False)
    return dt(x)


def _idiv(a, b):
    if isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
        a, b = np.asarray(a, np.int64), np.asarray(b, np.int64)
        return np.sign(a) * np.sign(b) * (np.abs(a) // np.abs(b))
    a, b = int(a), int(b)
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _ipow(x, n):
    """x**n for an integer n by repeated squaring, in x's own type."""
    if n == 0:
        return x * 0 + 1
    neg = n < 0
    n = abs(n)
    result = None
    base = x
    while n:
        if n & 1:
            result = base if result is None else result * base
        n >>= 1
        if n:
            base = base * base
    if neg:
        one = _conv(1, result.dtype.type) if isinstance(result, (np.ndarray, np.generic)) else 1.0
        return one / result
    return result


def arith(op, a, b):
    if op == "**":
        cb = _cat(b)
        if cb == "i" and not isinstance(b, np.ndarray):
            if _cat(a) == "i":
                return int(a) ** int(b) if int(b) >= 0 else _idiv(1, int(a) ** -int(b))
            return _ipow(a, int(b))
        dt = _result_dtype(a, b) or np.float64
        return np.power(_conv(a, dt), _conv(b, dt))
    dt = _result_dtype(a, b)
    if dt is None:
        if op == "+":
            return a + b
        if op == "-":
            return a - b
        if op == "*":
            return a * b
        if op == "/":
            return _idiv(a, b)
    a, b = _conv(a, dt), _conv(b, dt)
    if op == "+":
        return a + b
    if op == "-":
        return a - b
    if op == "*":
        return a * b
    if op == "/":
        return a / b
    raise FortranError(f"operator {op}")


def compare(op, a, b):
    if _cat(a) == "s" or _cat(b) == "s":
        a, b = str(a).rstrip(), str(b).rstrip()
    else:
        dt = _result_dtype(a, b)
        if dt is not None:
            a, b = _conv(a, dt), _conv(b, dt)
    r = {"==": np.equal, "/=": np.not_equal, "<": np.less, "<=": np.less_equal,
         ">": np.greater, ">=": np.greater_equal}[op](a, b)
    return bool(r) if not isinstance(r, np.ndarray) else r


def _logical(a):
    return a if isinstance(a, np.ndarray) else bool(a)


# ----------------------------------------------------------------------------
# signals


class _Goto(Exception):
    def __init__(self, label):
        self.label = label


class _Return(Exception):
    pass


class Stop(Exception):
    pass


# ----------------------------------------------------------------------------
# program units


class Decl:
    __slots__ = ("name", "type", "dims", "charlen", "is_param", "common")

    def __init__(self, name):
        self.name = name
        self.type = None
        self.dims = None       # list of (lo_ast, hi_ast or '*')
        self.charlen = None
        self.is_param = False
        self.common = None


class Unit:
    def __init__(self, kind, name, args, origin):
        self.kind, self.name, self.args, self.origin = kind, name, args, origin
        self.decls: dict[str, Decl] = {}
        self.params: list[tuple[str, object]] = []     # in order (name, ast)
        self.commons: list[tuple[str, list[str]]] = []
        self.implicit = {}
        self.implicit_none = False
        self.body = []              # list of (label, stmt-node, origin)
        self.data = []

    def decl(self, name):
        d = self.decls.get(name)
        if d is None:
            d = self.decls[name] = Decl(name)
        return d

    def type_of(self, name):
        d = self.decls.get(name)
        if d is not None and d.type is not None:
            return d.type
        if name in self.implicit:
            return self.implicit[name]
        if self.implicit_none:
            return None
        return "integer" if name[0] in "ijklmn" else "real"


_TYPE_RE = re.compile(r"^(integer|real|complex|logical|double\s*precision|character)"
                      r"(\s*\*\s*(\d+|\(\*\)|\(\s*\d+\s*\)))?\s*(?:,\s*|(?=\s)|(?=::))(.*)$")


def _type_norm(t, star):
    t = re.sub(r"\s+", " ", t)
    if t == "double precision":
        return "real8"
    if t == "real" and star and star.strip("*( )") == "8":
        return "real8"
    if t == "complex" and star and star.strip("*( )") in ("16",):
        return "complex16"
    return t


def _parse_entities(text):
    """Entities of a declaration: list of (name, dims-text or None, charlen)."""
    text = text.strip()
    if text.startswith("::"):
        text = text[2:]
    out = []
    for ent in split_top(text):
        if not ent:
            continue
        m = re.match(r"([a-z_][a-z0-9_]*)\s*(\(.*\))?\s*(\*\s*(\(\*\)|\d+))?\s*$", ent)
        if not m:
            raise FortranError(f"cannot parse declaration entity {ent!r}")
        dims = m.group(2)[1:-1] if m.group(2) else None
        out.append((m.group(1), dims, m.group(4)))
    return out


def _parse_dims(text):
    dims = []
    for d in split_top(text):
        if d == "*":
            dims.append((("lit", "n", "1"), "*"))
        elif ":" in d and d.count(":") == 1:
            lo, hi = d.split(":")
            dims.append((parse_expr(lo), "*" if hi.strip() == "*" else parse_expr(hi)))
        else:
            dims.append((("lit", "n", "1"), parse_expr(d)))
    return dims


def _parse_unit_header(text):
    m = re.match(r"^(subroutine|program)\s+([a-z_][a-z0-9_]*)\s*(\((.*)\))?\s*$", text)
    if not m:
        return None
    args = [a.strip() for a in m.group(4).split(",")] if m.group(4) and m.group(4).strip() else []
    return m.group(1), m.group(2), args


def split_units(stmts):
    units = []
    cur = None
    for lab, txt, org in stmts:
        if cur is None:
            h = _parse_unit_header(txt)
            if h is None:
                raise FortranError(f"{org}: statement outside a program unit: {txt!r}")
            cur = Unit(h[0], h[1], h[2], org)
            continue
        if re.match(r"^end(\s*(subroutine|program|function)(\s+[a-z0-9_]+)?)?$", txt):
            units.append(cur)
            cur = None
            continue
        cur.body.append((lab, txt, org))
    if cur is not None:
        raise FortranError(f"{cur.origin}: unit {cur.name} has no end")
    return units


def analyse_declarations(unit: Unit):
    """Move declaration statements out of the body into the unit's tables."""
    body = []
    for lab, txt, org in unit.body:
        try:
            if txt.startswith("implicit"):
                rest = txt[8:].strip()
                if rest == "none":
                    unit.implicit_none = True
                    continue
                m = re.match(r"^(integer|real|complex|logical|double\s*precision)\s*\((.*)\)$", rest)
                if not m:
                    raise FortranError(f"implicit statement {txt!r}")
                t = _type_norm(m.group(1), None)
                for rng in m.group(2).split(","):
                    a, _, b = rng.strip().partition("-")
                    b = b or a
                    for c in range(ord(a.strip()), ord(b.strip()) + 1):
                        unit.implicit[chr(c)] = t
                continue
            if txt.startswith("use ") or txt == "use mpi":
                unit.implicit.setdefault("__mpi__", True)
                continue
            if txt.startswith("intrinsic") or txt.startswith("external") or txt == "save":
                continue
            if txt.startswith("parameter"):
                inner = txt[txt.index("(") + 1: match_paren(txt, txt.index("("))]
                for item in split_top(inner):
                    name, _, val = item.partition("=")
                    name = name.strip()
                    unit.decl(name).is_param = True
                    unit.params.append((name, parse_expr(val)))
                continue
            if txt.startswith("common"):
                rest = txt[6:].strip()
                for m in re.finditer(r"/\s*([a-z0-9_]*)\s*/([^/]*)", rest):
                    names = []
                    for name, dims, _ in _parse_entities(m.group(2)):
                        if dims:
                            unit.decl(name).dims = _parse_dims(dims)
                        unit.decl(name).common = m.group(1)
                        names.append(name)
                    unit.commons.append((m.group(1), names))
                continue
            if txt.startswith("dimension"):
                for name, dims, _ in _parse_entities(txt[9:]):
                    unit.decl(name).dims = _parse_dims(dims)
                continue
            m = re.match(r"^(integer|real|complex|logical|double\s*precision)(\s*\*\s*\d+)?\s*,\s*(.*?)::(.*)$",
                         txt)
            if m:  # F90 form: type, attributes :: entities [= value]
                t = _type_norm(m.group(1), m.group(2))
                attrs = [x.strip() for x in split_top(m.group(3))]
                for ent in split_top(m.group(4)):
                    lhs, eq, val = ent.partition("=")
                    (name, dims, _), = _parse_entities(lhs)
                    d = unit.decl(name)
                    d.type = t
                    if dims:
                        d.dims = _parse_dims(dims)
                    if "parameter" in attrs:
                        d.is_param = True
                        unit.params.append((name, parse_expr(val)))
                continue
            m = _TYPE_RE.match(txt)
            if m and not re.match(r"^(real|integer|complex|logical)\s*\(", txt) and "=" not in txt.split("::")[0] \
                    or (m and "::" in txt):
                t = _type_norm(m.group(1), m.group(3))
                clen = None
                if t == "character":
                    s = (m.group(3) or "").strip("*( )")
                    clen = int(s) if s.isdigit() else 0
                for name, dims, elen in _parse_entities(m.group(4)):
                    d = unit.decl(name)
                    d.type = t
                    if t == "character":
                        d.charlen = int(elen) if elen and elen.isdigit() else clen
                    if dims:
                        d.dims = _parse_dims(dims)
                continue
        except FortranError as e:
            raise FortranError(f"{org}: {e}") from None
        body.append((lab, txt, org))
    unit.body = body


# ----------------------------------------------------------------------------
# statement parsing into a block tree


class Node:
    __slots__ = ("kind", "a", "origin", "label")

    def __init__(self, kind, a, origin, label=None):
        self.kind, self.a, self.origin, self.label = kind, a, origin, label


def _parse_io_control(text):
    """'(unit, fmt, err=20)' -> list of (key or None, value text)."""
    out = []
    for part in split_top(text):
        k, eq, v = part.partition("=")
        if eq and re.match(r"^[a-z_]+$", k.strip()):
            out.append((k.strip(), v.strip()))
        else:
            out.append((None, part.strip()))
    return out


def _parse_io_items(text):
    items = []
    for it in split_top(text):
        if not it:
            continue
        if it.startswith("(") and match_paren(it, 0) == len(it) - 1:
            inner = split_top(it[1:-1])
            if len(inner) >= 3 and re.match(r"^[a-z_][a-z0-9_]*\s*=", inner[-2]):
                var, _, lo = inner[-2].partition("=")
                items.append(("ido", _parse_io_items(",".join(inner[:-2])), var.strip(),
                              parse_expr(lo), parse_expr(inner[-1]), None))
                continue
        items.append(("item", parse_expr(it)))
    return items


def parse_simple(txt, org, lab):
    """One non-block statement."""
    if txt == "continue":
        return Node("continue", None, org, lab)
    if txt in ("return",):
        return Node("return", None, org, lab)
    if txt.startswith("stop"):
        return Node("stop", None, org, lab)
    m = re.match(r"^go\s*to\s*(\d+)$", txt)
    if m:
        return Node("goto", int(m.group(1)), org, lab)
    if txt.startswith("format"):
        return Node("continue", None, org, lab)
    m = re.match(r"^call\s+([a-z_][a-z0-9_]*)\s*(\((.*)\))?\s*$", txt)
    if m:
        args = []
        if m.group(2):
            inner = m.group(3)
            args = [_parse_arg(a) for a in split_top(inner)] if inner.strip() else []
        return Node("call", (m.group(1), args), org, lab)
    m = re.match(r"^(write|read|open|close|print)\s*\(", txt)
    if m:
        k = m.group(1)
        p0 = txt.index("(")
        p1 = match_paren(txt, p0)
        ctl = _parse_io_control(txt[p0 + 1:p1])
        items = _parse_io_items(txt[p1 + 1:].strip().lstrip(",")) if k in ("write", "read") else []
        return Node(k, (ctl, items), org, lab)
    m = re.match(r"^print\s", txt)
    if m:
        return Node("continue", None, org, lab)
    m = re.match(r"^where\s*\(", txt)
    if m:
        p1 = match_paren(txt, txt.index("("))
        mask = parse_expr(txt[txt.index("(") + 1:p1])
        inner = parse_simple(txt[p1 + 1:].strip(), org, None)
        return Node("where1", (mask, inner), org, lab)
    # assignment
    eq = _assign_split(txt)
    if eq is not None:
        lhs, rhs = eq
        return Node("assign", (parse_expr(lhs), parse_expr(rhs)), org, lab)
    raise FortranError(f"{org}: unsupported statement {txt!r}")


def _parse_arg(a):
    p = _P(a)
    e = p.arg()
    if p.peek()[0] != "end":
        raise FortranError(f"cannot parse argument {a!r}")
    return e


def _assign_split(txt):
    depth, q = 0, None
    for i, ch in enumerate(txt):
        if q:
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0:
            nxt = txt[i + 1] if i + 1 < len(txt) else ""
            prv = txt[i - 1] if i else ""
            if nxt == "=" or prv in "<>/=":
                return None
            return txt[:i].strip(), txt[i + 1:].strip()
    return None


class BlockParser:
    def __init__(self, stmts):
        self.s = stmts
        self.i = 0

    def parse_block(self, end_kinds=(), do_label=None):
        """Parse until a statement whose keyword is in end_kinds, or until the
        statement labelled do_label has been included.  Returns (nodes, end)."""
        nodes = []
        while self.i < len(self.s):
            lab, txt, org = self.s[self.i]
            key = self._end_key(txt)
            if key and key in end_kinds:
                self.i += 1
                return nodes, (key, txt, org, lab)
            self.i += 1
            node = self.parse_stmt(lab, txt, org)
            nodes.append(node)
            if do_label is not None and lab == do_label:
                return nodes, ("label", txt, org, lab)
            if isinstance(node, Node) and node.kind == "do" and node.a[-1] is not None and \
                    do_label is not None and node.a[-1] == do_label:
                # the inner DO shared this loop's terminating statement
                return nodes, ("label", txt, org, lab)
        if end_kinds or do_label is not None:
            raise FortranError(f"block not closed (expected {end_kinds or do_label})")
        return nodes, None

    @staticmethod
    def _end_key(txt):
        if re.match(r"^end\s*do$", txt):
            return "enddo"
        if re.match(r"^end\s*if$", txt):
            return "endif"
        if re.match(r"^else\s*if\s*\(", txt):
            return "elseif"
        if txt == "else":
            return "else"
        if re.match(r"^end\s*where$", txt):
            return "endwhere"
        if re.match(r"^else\s*where$", txt):
            return "elsewhere"
        return None

    def parse_stmt(self, lab, txt, org):
        m = re.match(r"^do\s+(\d+)?\s*,?\s*([a-z_][a-z0-9_]*)\s*=\s*(.*)$", txt)
        if m and len(split_top(m.group(3))) >= 2:
            label = int(m.group(1)) if m.group(1) else None
            bounds = [parse_expr(x) for x in split_top(m.group(3))]
            if label is None:
                body, _ = self.parse_block(("enddo",))
            else:
                body, _ = self.parse_block((), do_label=label)
            return Node("do", (m.group(2), bounds, body, label), org, lab)
        m = re.match(r"^if\s*\(", txt)
        if m:
            p0 = txt.index("(")
            p1 = match_paren(txt, p0)
            cond = parse_expr(txt[p0 + 1:p1])
            rest = txt[p1 + 1:].strip()
            if rest == "then":
                branches = []
                cur_cond = cond
                while True:
                    body, end = self.parse_block(("elseif", "else", "endif"))
                    branches.append((cur_cond, body))
                    key, etxt, eorg, _ = end
                    if key == "endif":
                        break
                    if key == "else":
                        body, _ = self.parse_block(("endif",))
                        branches.append((None, body))
                        break
                    q0 = etxt.index("(")
                    q1 = match_paren(etxt, q0)
                    cur_cond = parse_expr(etxt[q0 + 1:q1])
                return Node("if", branches, org, lab)
            return Node("if", [(cond, [parse_simple(rest, org, None)])], org, lab)
        m = re.match(r"^where\s*\((.*)\)\s*$", txt)
        if m and match_paren(txt, txt.index("(")) == len(txt) - 1:
            mask = parse_expr(txt[txt.index("(") + 1:-1])
            body, end = self.parse_block(("elsewhere", "endwhere"))
            other = []
            if end[0] == "elsewhere":
                other, _ = self.parse_block(("endwhere",))
            return Node("where", (mask, body, other), org, lab)
        return parse_simple(txt, org, lab)


# ----------------------------------------------------------------------------
# the interpreter


_MPI_PARAMS = {"mpi_comm_world": 91, "mpi_real": 1, "mpi_integer": 2, "mpi_complex": 3,
               "mpi_double_precision": 4, "mpi_logical": 5, "mpi_character": 6, "mpi_sum": 11,
               "mpi_max": 12, "mpi_min": 13, "mpi_status_size": 6, "mpi_double_complex": 7,
               "mpi_real8": 4, "mpi_address_kind": 8, "mpi_integer_kind": 4, "mpi_offset_kind": 8,
               "mpi_any_source": -1, "mpi_any_tag": -1, "mpi_success": 0, "mpi_datatype_null": 0,
               "mpi_lb": 0, "mpi_ub": 0, "mpi_comm_null": 0}


class Frame:
    __slots__ = ("unit", "vars", "params")

    def __init__(self, unit):
        self.unit = unit
        self.vars = {}
        self.params = {}


class Runner:
    """Holds the loaded units, COMMON storage, the uniform stream and I/O."""

    def __init__(self, files: list[str], include_dirs: list[str], real_kind: int = 8):
        self.kinds = Kinds(real_kind)
        self.units: dict[str, Unit] = {}
        for f in files:
            for u in split_units(read_fixed_form(f, include_dirs)):
                analyse_declarations(u)
                bp = BlockParser(u.body)
                nodes, end = bp.parse_block()
                u.tree = nodes
                u.labels = None
                if u.name in self.units:
                    raise FortranError(f"unit {u.name} defined twice ({u.origin})")
                self.units[u.name] = u
        self.commons: dict[str, list] = {}
        self.stream = None
        self.stream_pos = 0
        self.files_in: dict[str, list[str]] = {}
        self.unit_files: dict[int, str] = {}
        self.read_pos: dict[int, int] = {}
        self.captured: dict[int, list] = {}
        self.capture_units: set[int] = set()
        self.stubs: dict[str, object] = {}
        self._common_checked = set()
        self.init_commons()
        warnings.filterwarnings("ignore", category=np.exceptions.ComplexWarning)

    # ---- public helpers -------------------------------------------------
    def set_stream(self, uniforms):
        self.stream = np.asarray(uniforms, dtype=np.float64)
        self.stream_pos = 0

    def call(self, name, *args):
        """Call a subroutine with Python values; returns the (possibly
        updated) scalar arguments in order."""
        refs = []
        for a in args:
            if isinstance(a, (Ref, Arr, CharVar)):
                refs.append(a)
            elif isinstance(a, float):
                refs.append(Ref(np.array([a], self.kinds.real), 0))
            elif isinstance(a, int):
                refs.append(Ref(np.array([a], np.int64), 0))
            else:
                raise FortranError(f"argument of type {type(a)}")
        with np.errstate(all="ignore"):
            self._invoke(self.units[name], refs, name)
        return [r.get() if isinstance(r, Ref) else r for r in refs]

    def common_var(self, block, name):
        """The storage of a COMMON variable (Ref or Arr) by block and name."""
        for (n, v) in self.commons[block]:
            if n == name:
                return v
        raise KeyError(f"{name} not in /{block}/")

    # ---- storage --------------------------------------------------------
    def _dtype(self, t):
        k = self.kinds
        return {"integer": np.int64, "real": k.real, "real8": np.float64, "complex": k.cplx,
                "complex16": np.complex128, "logical": np.bool_}[t]

    def _fill(self, t):
        return {"integer": 0, "logical": False}.get(t, np.nan)

    def _new_storage(self, unit, frame, name, init_nan=True):
        d = unit.decls.get(name)
        t = unit.type_of(name)
        if t is None:
            raise FortranError(f"{unit.name}: {name} has no type (implicit none)")
        if t == "character":
            return CharVar(d.charlen if d else 0)
        dt = self._dtype(t)
        if d is not None and d.dims:
            lo, ext = self._eval_dims(d.dims, frame)
            n = int(np.prod(ext)) if ext else 1
            buf = np.full(n, self._fill(t) if init_nan else 0, dtype=dt)
            return Arr(buf, 0, lo, ext)
        return Ref(np.full(1, self._fill(t) if init_nan else 0, dtype=dt), 0)

    def _eval_dims(self, dims, frame, assumed_ok=False):
        lo, ext = [], []
        for lo_ast, hi_ast in dims:
            lv = int(self._eval(lo_ast, frame))
            if hi_ast == "*":
                if not assumed_ok:
                    raise FortranError("assumed-size array that is not a dummy argument")
                hv = lv
            else:
                hv = int(self._eval(hi_ast, frame))
            lo.append(lv)
            ext.append(max(hv - lv + 1, 0))
        return lo, ext

    def init_commons(self):
        """Create every COMMON block the loaded units declare (zeroed, like
        static storage at program start)."""
        for unit in self.units.values():
            self._frame_base(unit)

    def _setup_frame(self, unit, actuals):
        f = self._frame_base(unit)
        return self._bind(unit, f, actuals)

    def _frame_base(self, unit):
        f = Frame(unit)
        if unit.implicit.get("__mpi__"):
            f.params.update(_MPI_PARAMS)
        # mpif.h-style names may also be used without USE (include 'mpif.h' maps to it)
        for name, ast in unit.params:
            d = unit.decls.get(name)
            v = self._eval(ast, f)
            t = unit.type_of(name)
            if t == "character":
                f.params[name] = str(v)
            elif t is not None:
                f.params[name] = self._cast_scalar(v, t)
            else:
                f.params[name] = v
        # COMMON blocks
        for block, names in unit.commons:
            store = self.commons.get(block)
            if store is None:
                store = []
                for n in names:
                    store.append((n, self._new_storage(unit, f, n, init_nan=False)))
                self.commons[block] = store
            elif (unit.name, block) not in self._common_checked:
                self._common_checked.add((unit.name, block))
                if len(store) != len(names):
                    raise FortranError(f"{unit.name}: /{block}/ declared with a different layout")
                for (n0, v0), n in zip(store, names):
                    v1 = self._new_storage(unit, f, n, init_nan=False)
                    s0 = v0.size if isinstance(v0, Arr) else 1
                    s1 = v1.size if isinstance(v1, Arr) else 1
                    if type(v0) is not type(v1) or s0 != s1:
                        raise FortranError(f"{unit.name}: /{block}/ member {n} differs from {n0}")
            for (n0, v0), n in zip(store, names):
                f.vars[n] = v0
        return f

    def _bind(self, unit, f, actuals):
        # dummies: scalars first (they may size the arrays), then arrays
        if len(actuals) != len(unit.args):
            raise FortranError(f"{unit.name}: {len(actuals)} arguments for {len(unit.args)} dummies")
        pending = []
        for name, act in zip(unit.args, actuals):
            d = unit.decls.get(name)
            if d is not None and d.dims:
                pending.append((name, act, d))
            else:
                if isinstance(act, Arr):
                    f.vars[name] = Ref(act.buf, act.off)
                else:
                    f.vars[name] = act
        for name, act, d in pending:
            lo, ext = self._eval_dims(d.dims, f, assumed_ok=True)
            assumed = d.dims[-1][1] == "*"
            if isinstance(act, Arr):
                buf, off = act.buf, act.off
            elif isinstance(act, Ref):
                buf, off = act.buf, act.idx
            else:
                raise FortranError(f"{unit.name}: array dummy {name} given {type(act)}")
            want = self._dtype(unit.type_of(name))
            if buf.dtype != want:
                raise FortranError(f"{unit.name}: dummy {name} is {np.dtype(want)}, actual is {buf.dtype}")
            f.vars[name] = Arr(buf, off, lo, ext, assumed=assumed, dummy=True)
        # locals
        for name, d in unit.decls.items():
            if name in f.vars or name in f.params or d.is_param:
                continue
            if d.type is None and not d.dims:
                continue
            f.vars[name] = self._new_storage(unit, f, name)
        return f

    def _cast_scalar(self, v, t):
        if t == "character":
            return str(v)
        dt = self._dtype(t)
        if t == "integer":
            return int(np.trunc(np.real(v)))
        if t == "logical":
            return bool(v)
        return dt(v)

    def _var(self, frame, name):
        v = frame.vars.get(name)
        if v is not None:
            return v
        if name in frame.params:
            return None
        t = frame.unit.type_of(name)
        if t is None:
            raise FortranError(f"{frame.unit.name}: undeclared {name}")
        v = self._new_storage(frame.unit, frame, name)
        frame.vars[name] = v
        return v

    # ---- invocation -----------------------------------------------------
    def _invoke(self, unit, actuals, name):
        frame = self._setup_frame(unit, actuals)
        try:
            self._run_block(unit.tree, frame)
        except _Return:
            pass
        except _Goto as g:
            raise FortranError(f"{unit.name}: goto {g.label} has no target")

    def _run_block(self, nodes, frame):
        i = 0
        n = len(nodes)
        while i < n:
            node = nodes[i]
            try:
                self._exec(node, frame)
                i += 1
            except _Goto as g:
                for j, nd in enumerate(nodes):
                    if nd.label == g.label:
                        i = j
                        break
                else:
                    raise

    def _exec(self, node, frame):
        k = node.kind
        try:
            if k == "assign":
                self._assign(node.a[0], node.a[1], frame, None)
            elif k == "do":
                var, bounds, body, _ = node.a
                a = self._eval(bounds[0], frame)
                b = self._eval(bounds[1], frame)
                c = self._eval(bounds[2], frame) if len(bounds) > 2 else 1
                ref = self._var(frame, var)
                trips = max(_idiv(int(b) - int(a) + int(c), int(c)), 0)
                val = int(a)
                for _ in range(trips):
                    ref.set(val)
                    self._run_block(body, frame)
                    val = int(ref.get()) + int(c)
                ref.set(val)
            elif k == "if":
                for cond, body in node.a:
                    if cond is None or bool(self._eval(cond, frame)):
                        self._run_block(body, frame)
                        break
            elif k == "where":
                mask, body, other = node.a
                m = np.asarray(self._eval(mask, frame), dtype=bool)
                for st in body:
                    self._exec_masked(st, frame, m)
                for st in other:
                    self._exec_masked(st, frame, ~m)
            elif k == "where1":
                mask, inner = node.a
                m = np.asarray(self._eval(mask, frame), dtype=bool)
                self._exec_masked(inner, frame, m)
            elif k == "call":
                self._call(node.a[0], node.a[1], frame)
            elif k == "continue":
                pass
            elif k == "goto":
                raise _Goto(node.a)
            elif k == "return":
                raise _Return()
            elif k == "stop":
                raise Stop(node.origin)
            elif k == "write":
                self._write(node.a, frame)
            elif k == "read":
                self._read(node.a, frame)
            elif k == "open":
                self._open(node.a, frame)
            elif k in ("close", "print"):
                pass
            else:
                raise FortranError(f"statement kind {k}")
        except (FortranError, ValueError, TypeError, IndexError, KeyError) as e:
            if getattr(e, "_located", False):
                raise
            err = FortranError(f"{node.origin} ({frame.unit.name}): {e}")
            err._located = True
            raise err from None

    def _exec_masked(self, st, frame, mask):
        if st.kind != "assign":
            raise FortranError(f"{st.origin}: only assignments inside WHERE")
        self._assign(st.a[0], st.a[1], frame, mask)

    # ---- assignment -----------------------------------------------------
    def _assign(self, lhs, rhs, frame, mask):
        val = self._eval(rhs, frame)
        if lhs[0] == "name":
            target = self._var(frame, lhs[1])
            if target is None:
                raise FortranError(f"assignment to parameter {lhs[1]}")
            if isinstance(target, Arr):
                view = target.view()
                self._store_view(view, val, mask)
            else:
                if mask is not None:
                    raise FortranError("scalar assignment under a WHERE mask")
                if isinstance(target, CharVar):
                    target.set(val)
                else:
                    target.set(self._scalar_for(target.buf.dtype, val))
            return
        if lhs[0] == "ref":
            target = self._var(frame, lhs[1])
            if not isinstance(target, Arr):
                raise FortranError(f"{lhs[1]} is not an array")
            subs = [self._eval_sub(s, frame) for s in lhs[2]]
            if all(not isinstance(s, slice) for s in subs):
                if mask is not None:
                    raise FortranError("element assignment under a WHERE mask")
                target.buf[target.index(subs)] = self._scalar_for(target.buf.dtype, val)
                return
            view = target.view()[self._np_index(target, subs)]
            self._store_view(view, val, mask)
            return
        raise FortranError(f"cannot assign to {lhs}")

    @staticmethod
    def _scalar_for(dt, val):
        if isinstance(val, np.ndarray):
            raise FortranError("array value assigned to a scalar")
        if dt.kind in "iu":
            return int(np.trunc(np.real(val)))
        if dt.kind == "f":
            return np.real(val)
        return val

    @staticmethod
    def _store_view(view, val, mask):
        if isinstance(val, np.ndarray) and val.dtype.kind == "c" and view.dtype.kind != "c":
            val = val.real
        elif not isinstance(val, np.ndarray) and view.dtype.kind == "f":
            val = np.real(val)
        if mask is None:
            view[...] = val
        else:
            full = np.broadcast_to(np.asarray(val), view.shape)
            view[mask] = full[mask]

    def _np_index(self, arr, subs):
        idx = []
        for s, lo, e in zip(subs, arr.lo, arr.ext):
            if isinstance(s, slice):
                a = lo if s.start is None else s.start
                b = lo + e - 1 if s.stop is None else s.stop
                st = 1 if s.step is None else s.step
                if st != 1:
                    raise FortranError("strided sections are not supported")
                if a < lo or b > lo + e - 1:
                    raise FortranError("section out of bounds")
                idx.append(slice(a - lo, b - lo + 1))
            else:
                r = int(s) - lo
                if r < 0 or r >= e:
                    raise FortranError(f"subscript {int(s)} out of bounds")
                idx.append(r)
        return tuple(idx)

    def _eval_sub(self, s, frame):
        if isinstance(s, tuple) and s[0] == "sec":
            lo = None if s[1] is None else int(self._eval(s[1], frame))
            hi = None if s[2] is None else int(self._eval(s[2], frame))
            st = None if s[3] is None else int(self._eval(s[3], frame))
            return slice(lo, hi, st)
        return int(self._eval(s, frame))

    # ---- expressions ----------------------------------------------------
    def _lit(self, node):
        kind, txt = node[1], node[2]
        if kind == "l":
            return bool(txt)
        if kind == "s":
            return txt
        if re.fullmatch(r"\d+", txt):
            return int(txt)
        if "d" in txt:
            return np.float64(float(txt.replace("d", "e")))
        return self.kinds.real(float(txt))

    def _eval(self, node, frame):
        k = node[0]
        if k == "lit":
            return self._lit(node)
        if k == "name":
            name = node[1]
            if name in frame.params:
                return frame.params[name]
            v = self._var(frame, name)
            if isinstance(v, Arr):
                return v.view()
            return v.get()
        if k == "bin":
            op = node[1]
            a = self._eval(node[2], frame)
            b = self._eval(node[3], frame)
            if op in ("+", "-", "*", "/", "**"):
                return arith(op, a, b)
            if op in ("==", "/=", "<", "<=", ">", ">="):
                return compare(op, a, b)
            if op == ".and.":
                return np.logical_and(a, b) if isinstance(a, np.ndarray) or isinstance(b, np.ndarray) \
                    else bool(a) and bool(b)
            if op == ".or.":
                return np.logical_or(a, b) if isinstance(a, np.ndarray) or isinstance(b, np.ndarray) \
                    else bool(a) or bool(b)
            if op == ".eqv.":
                return compare("==", _logical(a), _logical(b))
            if op == ".neqv.":
                return compare("/=", _logical(a), _logical(b))
            if op == "//":
                return str(a) + str(b)
            raise FortranError(f"operator {op}")
        if k == "neg":
            return -self._eval(node[1], frame)
        if k == "not":
            v = self._eval(node[1], frame)
            return np.logical_not(v) if isinstance(v, np.ndarray) else not bool(v)
        if k == "paren":
            return self._eval(node[1], frame)
        if k == "cmplx_lit":
            re_ = self._eval(node[1], frame)
            im_ = self._eval(node[2], frame)
            dt = _result_dtype(re_, im_) or self.kinds.real
            return (np.complex128 if dt in (np.float64, np.complex128) else np.complex64)(complex(re_, im_))
        if k == "arrcons":
            vals = [self._eval(x, frame) for x in node[1]]
            return np.array(vals)
        if k == "ref":
            return self._eval_ref(node, frame)
        raise FortranError(f"expression node {k}")

    def _eval_ref(self, node, frame):
        name, args = node[1], node[2]
        v = frame.vars.get(name)
        if v is None and name not in frame.params:
            d = frame.unit.decls.get(name)
            if d is not None and d.dims:
                v = self._var(frame, name)
        if isinstance(v, Arr):
            subs = [self._eval_sub(s, frame) for s in args]
            if all(not isinstance(s, slice) for s in subs):
                return v.buf[v.index(subs)]
            return v.view()[self._np_index(v, subs)]
        return self._intrinsic(name, args, frame)

    # ---- intrinsics -----------------------------------------------------
    def _intrinsic(self, name, args, frame):
        ev = [self._eval(a, frame) for a in args if not (isinstance(a, tuple) and a[0] == "kw")]
        kw = {a[1]: self._eval(a[2], frame) for a in args if isinstance(a, tuple) and a[0] == "kw"}
        K = self.kinds
        if name in ("sqrt", "exp", "log", "cos", "sin", "acos", "asin", "atan", "tan", "log10"):
            x = ev[0]
            if _cat(x) == "i":
                raise FortranError(f"{name} of an integer")
            fn = {"sqrt": np.sqrt, "exp": np.exp, "log": np.log, "cos": np.cos, "sin": np.sin,
                  "acos": np.arccos, "asin": np.arcsin, "atan": np.arctan, "tan": np.tan,
                  "log10": np.log10}[name]
            return fn(x)
        if name == "atan2":
            dt = _result_dtype(ev[0], ev[1])
            return np.arctan2(_conv(ev[0], dt), _conv(ev[1], dt))
        if name == "abs":
            x = ev[0]
            return abs(x) if _cat(x) == "i" and not isinstance(x, np.ndarray) else np.abs(x)
        if name in ("real", "float", "sngl", "dble"):
            x = ev[0]
            kind = kw.get("kind", ev[1] if len(ev) > 1 else None)
            if name == "dble" or kind == 8:
                dt = np.float64
            elif _cat(x) == "c" and name == "real" and kind is None:
                return np.real(x)
            else:
                dt = K.real
            return _conv(np.real(x), dt)
        if name == "aimag":
            return np.imag(ev[0])
        if name == "conjg":
            return np.conj(ev[0])
        if name == "cmplx":
            re_ = ev[0]
            im_ = ev[1] if len(ev) > 1 else 0
            kind = kw.get("kind", ev[2] if len(ev) > 2 else None)
            dt = np.complex128 if kind == 8 else K.cplx
            rdt = np.float64 if dt == np.complex128 else np.float32
            if isinstance(re_, np.ndarray) or isinstance(im_, np.ndarray):
                out = np.empty(np.broadcast(re_, im_).shape, dt)
                out.real = _conv(np.real(re_), rdt)
                out.imag = _conv(np.real(im_), rdt)
                return out
            return dt(complex(rdt(np.real(re_)), rdt(np.real(im_))))
        if name == "aint":
            return np.trunc(ev[0])
        if name == "int":
            x = ev[0]
            return np.trunc(np.real(x)).astype(np.int64) if isinstance(x, np.ndarray) else int(np.trunc(np.real(x)))
        if name == "nint":
            x = ev[0]
            r = np.sign(x) * np.floor(np.abs(x) + 0.5)
            return r.astype(np.int64) if isinstance(r, np.ndarray) else int(r)
        if name == "mod":
            a, b = ev
            if _cat(a) == "i" and _cat(b) == "i":
                return arith("-", a, arith("*", _idiv(a, b), b))
            dt = _result_dtype(a, b)
            a, b = _conv(a, dt), _conv(b, dt)
            return np.fmod(a, b)
        if name == "sign":
            a, b = ev
            if _cat(a) == "i" and _cat(b) == "i":
                return abs(int(a)) if int(b) >= 0 else -abs(int(a))
            return np.copysign(np.abs(a), b)
        if name in ("min", "max"):
            if all(_cat(x) == "i" for x in ev):
                return (min if name == "min" else max)(int(x) for x in ev)
            dt = ev[0]
            for x in ev[1:]:
                dt = np.minimum(dt, x) if name == "min" else np.maximum(dt, x)
            return dt
        if name == "sum":
            x = np.asarray(ev[0])
            if x.size == 0:
                return x.dtype.type(0)
            return np.cumsum(x.ravel(order="F"), dtype=x.dtype)[-1]
        if name == "count":
            return int(np.count_nonzero(ev[0]))
        if name == "dot_product":
            a, b = np.asarray(ev[0]), np.asarray(ev[1])
            if a.dtype.kind == "c":
                a = np.conj(a)
            dt = _result_dtype(a, b) or np.int64
            p = (_conv(a, dt) * _conv(b, dt)).ravel(order="F")
            return np.cumsum(p, dtype=p.dtype)[-1]
        if name == "mpi_wtime":
            return np.float64(0.0)
        if name == "size":
            return int(np.asarray(ev[0]).size)
        if name in self.stubs:
            return self.stubs[name](*ev)
        raise FortranError(f"unknown function or array {name}")

    # ---- calls ----------------------------------------------------------
    def _actual(self, a, frame):
        """Bind an actual argument: a storage location for names and
        elements, a temporary for expressions."""
        if a[0] == "name":
            name = a[1]
            if name not in frame.params:
                v = self._var(frame, name)
                if v is not None:
                    return v
        if a[0] == "ref":
            v = frame.vars.get(a[1])
            if v is None and a[1] not in frame.params:
                d = frame.unit.decls.get(a[1])
                if d is not None and d.dims:
                    v = self._var(frame, a[1])
            if isinstance(v, Arr):
                subs = [self._eval_sub(s, frame) for s in a[2]]
                if any(isinstance(s, slice) for s in subs):
                    sec = v.view()[self._np_index(v, subs)]
                    if not (sec.flags.f_contiguous and np.shares_memory(sec, v.buf)):
                        raise FortranError("non-contiguous section passed as an argument")
                    off = v.off + (sec.__array_interface__["data"][0] -
                                   v.buf.__array_interface__["data"][0]) // v.buf.itemsize - v.off
                    return Arr(v.buf, off, [1] * sec.ndim, list(sec.shape))
                return Ref(v.buf, v.index(subs))
        val = self._eval(a, frame)
        if isinstance(val, np.ndarray):
            buf = np.array(val.ravel(order="F"))
            return Arr(buf, 0, [1] * val.ndim, list(val.shape))
        if isinstance(val, str):
            c = CharVar(0)
            c.set(val)
            return c
        if _cat(val) == "i":
            return Ref(np.array([int(val)], np.int64), 0)
        if _cat(val) == "l":
            return Ref(np.array([bool(val)]), 0)
        return Ref(np.array([val]), 0)

    def _call(self, name, args, frame):
        acts = [self._actual(a, frame) for a in args if not (isinstance(a, tuple) and a[0] == "kw")]
        kws = {a[1]: a[2] for a in args if isinstance(a, tuple) and a[0] == "kw"}
        if name in self.units:
            self._invoke(self.units[name], acts, name)
            return
        if name == "random_number":
            tgt = acts[0]
            if isinstance(tgt, Arr):
                n = tgt.size
                vals = self._draw(n)
                tgt.view()[...] = vals.reshape(tgt.ext, order="F")
            else:
                tgt.set(self._draw(1)[0])
            return
        if name in ("random_seed", "flush", "mpi_init", "mpi_finalize", "mpi_barrier", "mpi_bcast",
                    "mpi_wait", "mpi_type_commit", "mpi_type_vector", "mpi_type_create_struct",
                    "mpi_type_struct", "mpi_get_address", "mpi_type_get_extent", "mpi_type_free",
                    "mpi_comm_free", "mpi_address", "mpi_type_extent", "mpi_type_contiguous",
                    "mpi_type_indexed", "mpi_type_hvector", "mpi_type_create_resized"):
            return
        if name in ("mpi_issend", "mpi_irecv", "mpi_send", "mpi_recv", "mpi_isend", "mpi_sendrecv"):
            raise FortranError(f"{name} reached with one rank")
        if name in ("abort", "mpi_abort", "exit"):
            raise Stop(f"{name} called")
        if name == "mpi_comm_rank":
            acts[1].set(0)
            return
        if name == "mpi_comm_size":
            acts[1].set(1)
            return
        if name == "mpi_cart_create":
            acts[5].set(92)
            return
        if name == "mpi_cart_shift":
            acts[3].set(0)
            acts[4].set(0)
            return
        if name == "mpi_cart_coords":
            c = acts[3]
            if isinstance(c, Arr):
                c.view()[...] = 0
            else:
                c.set(0)
            return
        if name == "mpi_cart_sub":
            acts[2].set(93)
            return
        if name == "mpi_cartdim_get":
            acts[1].set(1)
            return
        if name == "mpi_cart_get":
            if isinstance(acts[2], Arr):
                acts[2].view()[...] = 1
            for k in (3, 4):
                t = acts[k]
                if isinstance(t, Arr):
                    t.view()[...] = 0 if t.buf.dtype.kind != "b" else True
                else:
                    t.set(0)
            return
        if name == "mpi_cart_rank":
            acts[2].set(0)
            return
        if name in ("mpi_reduce", "mpi_allreduce", "mpi_gather", "mpi_allgather"):
            send, recv = acts[0], acts[3] if name in ("mpi_gather", "mpi_allgather") else acts[1]
            count = int((acts[1] if name in ("mpi_gather", "mpi_allgather") else acts[2]).get())
            sb, so = (send.buf, send.off) if isinstance(send, Arr) else (send.buf, send.idx)
            rb, ro = (recv.buf, recv.off) if isinstance(recv, Arr) else (recv.buf, recv.idx)
            if sb.dtype != rb.dtype:
                raise FortranError(f"{name}: send {sb.dtype} and receive {rb.dtype} differ")
            rb[ro:ro + count] = sb[so:so + count].copy()
            return
        if name in self.stubs:
            self.stubs[name](*acts)
            return
        raise FortranError(f"call of unknown subroutine {name}")

    def _draw(self, n):
        if self.stream is None:
            raise FortranError("random_number called without a stream")
        if self.stream_pos + n > len(self.stream):
            raise FortranError("the uniform stream is exhausted")
        v = self.stream[self.stream_pos:self.stream_pos + n]
        self.stream_pos += n
        return v

    # ---- I/O ------------------------------------------------------------
    def _unit_of(self, ctl, frame):
        for k, v in ctl:
            if k in (None, "unit"):
                if v == "*":
                    return None
                u = self._eval(parse_expr(v), frame)
                return None if isinstance(u, str) else int(u)
        return None

    def _open(self, a, frame):
        ctl, _ = a
        unit = self._unit_of(ctl, frame)
        fname = None
        for k, v in ctl:
            if k == "file":
                fname = str(self._eval(parse_expr(v), frame)).strip()
        if unit is not None and fname is not None:
            self.unit_files[unit] = fname
            self.read_pos[unit] = 0

    def _items_values(self, items, frame, out):
        for it in items:
            if it[0] == "item":
                v = self._eval(it[1], frame)
                if isinstance(v, np.ndarray):
                    out.extend(v.ravel(order="F").tolist())
                else:
                    out.append(v.item() if isinstance(v, np.generic) else v)
            else:
                _, sub, var, lo, hi, _ = it
                ref = self._var(frame, var)
                for i in range(int(self._eval(lo, frame)), int(self._eval(hi, frame)) + 1):
                    ref.set(i)
                    self._items_values(sub, frame, out)

    def _write(self, a, frame):
        ctl, items = a
        unit = self._unit_of(ctl, frame)
        if unit is None or unit not in self.capture_units:
            return
        vals = []
        self._items_values(items, frame, vals)
        self.captured.setdefault(unit, []).append(vals)

    def _read(self, a, frame):
        ctl, items = a
        unit = self._unit_of(ctl, frame)
        fname = self.unit_files.get(unit)
        if fname not in self.files_in:
            raise FortranError(f"read from unit {unit} ({fname}) with no content")
        lines = self.files_in[fname]
        targets = []
        for it in items:
            if it[0] != "item":
                raise FortranError("implied-do in READ")
            targets.append(it[1])
        toks = []
        while len(toks) < len(targets):
            pos = self.read_pos[unit]
            if pos >= len(lines):
                raise FortranError(f"end of file {fname}")
            self.read_pos[unit] = pos + 1
            toks.extend(t for t in re.split(r"[,\s]+", lines[pos].strip()) if t)
        for tgt, tok in zip(targets, toks):
            if tgt[0] == "name":
                v = self._var(frame, tgt[1])
            else:
                arr = self._var(frame, tgt[1])
                v = Ref(arr.buf, arr.index([self._eval_sub(s, frame) for s in tgt[2]]))
            if isinstance(v, CharVar):
                v.set(tok.strip("'\""))
            elif v.buf.dtype.kind in "iu":
                v.set(int(tok))
            else:
                v.set(float(tok.lower().replace("d", "e")))
