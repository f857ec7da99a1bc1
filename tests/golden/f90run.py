"""Run the reference's Fortran 90 time loop on small lattices (test infrastructure).

The reference is five single-file Fortran 90 programs and no Fortran compiler
exists in this image, so this module translates the subset of Fortran those
programs use into Python and executes it, with the arithmetic semantics of
gfortran on x86-64 without -ffast-math:

  * default REAL literals (``0.05``, ``1.``, ``1.0E8``) are single precision;
    ``D`` exponents are double; an operation on two REAL(4) operands rounds to
    single (numpy float32), mixed operations widen to double first;
  * integer division truncates toward zero; ``x**n`` with a literal integer
    n is a product of n factors ((x*x)*x, as gfortran expands it);
  * ``SUM`` adds in array-element order (first index fastest), one term at
    a time; SQRT/SIN/COS/EXP of doubles are the C library's;
  * scalar arguments are passed by value-result, arrays and derived-type
    objects by reference;
  * local variables of subprograms keep their values between calls (static
    storage, zero at program start), which is how the reference's
    ``D_PW`` test in ComputeCollisionForce sees the previous call's value.

Input/output: list-directed READ takes numbers from in-memory file contents,
WRITE records its values per unit (the reference's time-history and
mean-density files become lists of numbers), PRINT/PAUSE/OPEN/CLOSE do
nothing, and subroutines named in ``stubs`` (the Tecplot writers) are not
executed.  PARAMETER values can be overridden before the module is
evaluated, which is how a run is shrunk to a small lattice and a few steps.

Only what the shipped programs use is supported; anything else raises
FortranError naming the statement.
"""

from __future__ import annotations

import ctypes
import math
import re

import numpy as np

__all__ = ["FortranError", "run_program"]


class FortranError(Exception):
    pass


class _Stop(Exception):
    def __init__(self, frame):
        super().__init__("STOP")
        self.frame = frame


# ----------------------------------------------------------------------------
# source -> statements
# ----------------------------------------------------------------------------

def _strip_comment(line: str) -> str:
    out, q = [], None
    for ch in line:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        elif ch == "!":
            break
        else:
            out.append(ch)
    return "".join(out)


def _split_semicolons(s: str):
    parts, cur, q = [], [], None
    for ch in s:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur.append(ch)
        elif ch == ";":
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur))
    return [p.strip() for p in parts if p.strip()]


def _upper_outside_quotes(s: str) -> str:
    out, q = [], None
    for ch in s:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        else:
            out.append(ch.upper())
    return "".join(out)


def read_statements(text: str):
    """(line number, statement) pairs: comments removed, continuation lines
    joined, ';'-separated statements split, upper-cased outside strings."""
    lines = text.replace("\r\n", "\n").replace("\r", "\n").split("\n")
    stmts = []
    buf, start = "", None
    for n, raw in enumerate(lines, 1):
        s = _strip_comment(raw.replace("\t", " ")).rstrip()
        if not s.strip():
            if buf:
                continue
            continue
        t = s.strip()
        if buf:
            if t.startswith("&"):
                t = t[1:]
            buf += t
        else:
            buf, start = t, n
        if buf.endswith("&"):
            buf = buf[:-1]
            continue
        for st in _split_semicolons(buf):
            stmts.append((start, _upper_outside_quotes(st)))
        buf = ""
    return stmts


# ----------------------------------------------------------------------------
# expressions
# ----------------------------------------------------------------------------

_TOK = re.compile(
    r"""\s*(?:
      (?P<str>'[^']*'|"[^"]*")
    | (?P<num>(?:\d+\.(?![A-Z]+\.)\d*|\.\d+|\d+)(?:[EDQ][+-]?\d+)?)
    | (?P<dot>\.(?:AND|OR|NOT|EQ|NE|LT|LE|GT|GE|TRUE|FALSE|EQV|NEQV)\.)
    | (?P<id>[A-Z_][A-Z0-9_]*)
    | (?P<op>\*\*|==|/=|<=|>=|//|\(/|/\)|::|[-+*/(),:%=<>])
    )""",
    re.X,
)


def tokenize(s: str):
    toks, pos = [], 0
    s = s.rstrip()
    while pos < len(s):
        m = _TOK.match(s, pos)
        if not m or m.end() == pos:
            raise FortranError(f"cannot tokenize: {s[pos:]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        toks.append((kind, m.group(kind)))
    return toks


class _P:
    """Recursive-descent parser over a token list."""

    def __init__(self, toks, src):
        self.t, self.i, self.src = toks, 0, src

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise FortranError(f"expected {val!r}, got {tok[1]!r} in {self.src!r}")
        self.i += 1
        return tok

    def at(self, val):
        return self.peek()[1] == val

    def done(self):
        return self.i >= len(self.t)

    # precedence climbing ---------------------------------------------------
    def expr(self):
        a = self.or_()
        while self.peek()[1] in (".EQV.", ".NEQV."):
            op = self.take()[1]
            a = ("op", op, a, self.or_())
        return a

    def or_(self):
        a = self.and_()
        while self.at(".OR."):
            self.take()
            a = ("op", ".OR.", a, self.and_())
        return a

    def and_(self):
        a = self.not_()
        while self.at(".AND."):
            self.take()
            a = ("op", ".AND.", a, self.not_())
        return a

    def not_(self):
        if self.at(".NOT."):
            self.take()
            return ("not", self.not_())
        return self.rel()

    _REL = {"==": "==", ".EQ.": "==", "/=": "!=", ".NE.": "!=", "<": "<", ".LT.": "<",
            "<=": "<=", ".LE.": "<=", ">": ">", ".GT.": ">", ">=": ">=", ".GE.": ">="}

    def rel(self):
        a = self.add()
        if self.peek()[1] in self._REL:
            op = self._REL[self.take()[1]]
            a = ("op", op, a, self.add())
        return a

    def add(self):
        if self.peek()[1] in ("+", "-"):
            sign = self.take()[1]
            a = self.mul()
            if sign == "-":
                a = ("neg", a)
        else:
            a = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = ("op", op, a, self.mul())
        return a

    def mul(self):
        a = self.unary_factor()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            a = ("op", op, a, self.unary_factor())
        return a

    def unary_factor(self):
        # gfortran accepts a sign after * and / (a*-b)
        if self.peek()[1] in ("+", "-"):
            sign = self.take()[1]
            f = self.power()
            return ("neg", f) if sign == "-" else f
        return self.power()

    def power(self):
        a = self.primary()
        if self.at("**"):
            self.take()
            b = self.unary_factor()  # right associative
            a = ("op", "**", a, b)
        return a

    def primary(self):
        kind, val = self.peek()
        if kind == "num":
            self.take()
            return _num_node(val)
        if kind == "str":
            self.take()
            return ("str", val[1:-1])
        if kind == "dot" and val in (".TRUE.", ".FALSE."):
            self.take()
            return ("log", val == ".TRUE.")
        if val == "(/":
            self.take()
            items = [self.expr()]
            while self.at(","):
                self.take()
                items.append(self.expr())
            self.take("/)")
            return ("ctor", items)
        if val == "(":
            self.take()
            e = self.expr()
            self.take(")")
            return ("paren", e)
        if kind == "id":
            self.take()
            node = ("name", val)
            while True:
                if self.at("("):
                    self.take()
                    args = []
                    if not self.at(")"):
                        args.append(self.arg())
                        while self.at(","):
                            self.take()
                            args.append(self.arg())
                    self.take(")")
                    node = ("ref", node, args)
                elif self.at("%"):
                    self.take()
                    node = ("comp", node, self.take()[1])
                else:
                    break
            return node
        raise FortranError(f"unexpected {val!r} in {self.src!r}")

    def arg(self):
        # subscript, section (lo:hi), or keyword argument is not used
        if self.at(":"):
            self.take()
            hi = None if (self.at(",") or self.at(")")) else self.expr()
            return ("slice", None, hi)
        e = self.expr()
        if self.at(":"):
            self.take()
            hi = None if (self.at(",") or self.at(")")) else self.expr()
            return ("slice", e, hi)
        return e


def _num_node(text: str):
    if re.fullmatch(r"\d+", text):
        return ("num", int(text), "i")
    if "D" in text:
        return ("num", float(text.replace("D", "E")), "r8")
    return ("num", text, "r4")  # keep the decimal text: rounded once to binary32


def parse_expr(s: str):
    p = _P(tokenize(s), s)
    e = p.expr()
    if not p.done():
        raise FortranError(f"trailing tokens in {s!r}")
    return e


# ----------------------------------------------------------------------------
# runtime helpers used by generated code
# ----------------------------------------------------------------------------

_f32 = np.float32
_libm = ctypes.CDLL("libm.so.6")
for _fn in ("sinf", "cosf", "expf", "sqrtf"):
    getattr(_libm, _fn).restype = ctypes.c_float
    getattr(_libm, _fn).argtypes = [ctypes.c_float]


def _idiv(a, b):
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _imod(a, b):
    return a - _idiv(a, b) * b


def _nint(x):
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def _seqsum(a):
    a = np.asarray(a)
    if a.size == 0:
        return 0.0 if a.dtype.kind == "f" else 0
    return np.add.accumulate(a.ravel(order="F"))[-1].item() if a.dtype == np.float64 else \
        np.add.accumulate(a.ravel(order="F"))[-1]


def _r4fn(name, x):
    return _f32(getattr(_libm, name)(float(x)))


def _powi(x, n):
    # gfortran expands x**n (integer literal n) into multiplications
    if n == 0:
        return 1
    if n < 0:
        return 1 / _powi(x, -n)
    if n == 1:
        return x
    if n == 2:
        return x * x
    if n == 3:
        return x * x * x
    h = _powi(x, n // 2)
    return h * h if n % 2 == 0 else h * h * x


class _IO:
    def __init__(self, files):
        self.files = dict(files or {})
        self.units = {}      # unit -> file name
        self.readers = {}    # unit -> [records, position]
        self.written = {}    # unit -> list of records (lists of values)

    def open(self, unit, name):
        self.units[unit] = name
        if name in self.files:
            recs = [r.replace(",", " ").split() for r in self.files[name].replace("\r", "").split("\n")]
            self.readers[unit] = [recs, 0]

    def read(self, unit, count):
        """count values from the next record(s) (list-directed)."""
        if unit not in self.readers:
            raise FortranError(f"READ from unit {unit} without input data")
        recs, pos = self.readers[unit]
        vals = []
        while len(vals) < count:
            if pos >= len(recs):
                raise FortranError(f"end of file on unit {unit}")
            vals.extend(recs[pos])
            pos += 1
        self.readers[unit][1] = pos
        return [float(v.replace("D", "E").replace("d", "e")) for v in vals[:count]]

    def write(self, unit, values):
        flat = []
        for v in values:
            if isinstance(v, np.ndarray):
                flat.extend(v.ravel(order="F").tolist())
            elif isinstance(v, str):
                continue
            else:
                flat.append(v.item() if hasattr(v, "item") else v)
        self.written.setdefault(unit, []).append(flat)


# ----------------------------------------------------------------------------
# symbols and types
# ----------------------------------------------------------------------------

_TYPE_KW = re.compile(
    r"^(DOUBLE\s*PRECISION|REAL\s*\*\s*8|REAL\s*\(\s*(?:KIND\s*=\s*)?8\s*\)|REAL\s*\(\s*(?:KIND\s*=\s*)?4\s*\)|"
    r"REAL|INTEGER|LOGICAL|CHARACTER\s*(?:\([^)]*\))?|TYPE\s*\(\s*([A-Z_][A-Z0-9_]*)\s*\))(?=[\s,:]|$)(.*)$")

_RANK = {"i": 0, "r4": 1, "r8": 2}


def _base_type(kw):
    kw = re.sub(r"\s+", "", kw)
    if kw.startswith("DOUBLEPRECISION") or kw in ("REAL*8", "REAL(8)", "REAL(KIND=8)"):
        return "r8"
    if kw.startswith("REAL"):
        return "r4"
    if kw == "INTEGER":
        return "i"
    if kw == "LOGICAL":
        return "l"
    if kw.startswith("CHARACTER"):
        return "c"
    raise FortranError(kw)


class Sym:
    def __init__(self, name, typ, dims=None, param=False, where="local", init=None):
        self.name, self.typ, self.dims = name, typ, dims  # dims: list of (lo, hi) exprs/ints
        self.param, self.where, self.init = param, where, init
        self.lbs = None  # lower bounds (ints) once known
        self.value = None  # evaluated PARAMETER value


def _split_top(s, sep=","):
    out, depth, cur, q = [], 0, [], None
    i = 0
    while i < len(s):
        ch = s[i]
        if q:
            cur.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur.append(ch)
        elif ch == "(":
            depth += 1
            cur.append(ch)
        elif ch == ")":
            depth -= 1
            cur.append(ch)
        elif ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
        i += 1
    out.append("".join(cur))
    return [x.strip() for x in out if x.strip()]


def _find_top(s, ch):
    depth, q = 0, None
    for i, c in enumerate(s):
        if q:
            if c == q:
                q = None
        elif c in "'\"":
            q = c
        elif c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        elif depth == 0 and s.startswith(ch, i):
            return i
    return -1


def _matching_paren(s, i):
    depth = 0
    for j in range(i, len(s)):
        if s[j] == "(":
            depth += 1
        elif s[j] == ")":
            depth -= 1
            if depth == 0:
                return j
    raise FortranError(f"unbalanced parentheses in {s!r}")


def _assign_pos(s):
    """index of the top-level '=' of an assignment, or -1."""
    depth, q = 0, None
    for i, c in enumerate(s):
        if q:
            if c == q:
                q = None
            continue
        if c in "'\"":
            q = c
        elif c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        elif c == "=" and depth == 0:
            prev = s[i - 1] if i else ""
            nxt = s[i + 1] if i + 1 < len(s) else ""
            if prev in "<>=/" or nxt == "=":
                continue
            return i
    return -1


def _parse_entity(e):
    """NAME[(dims)][=init] -> (name, [dim strings] or None, init string or None)."""
    init = None
    k = _assign_pos(e)
    if k >= 0:
        init = e[k + 1:].strip()
        e = e[:k].strip()
    m = re.match(r"^([A-Z_][A-Z0-9_]*)\s*(\((.*)\))?$", e)
    if not m:
        raise FortranError(f"bad entity {e!r}")
    dims = _split_top(m.group(3)) if m.group(2) else None
    return m.group(1), dims, init


# ----------------------------------------------------------------------------
# program units
# ----------------------------------------------------------------------------

class Unit:
    def __init__(self, kind, name, args, stmts, rtype=None):
        self.kind, self.name, self.args, self.stmts = kind, name, args, stmts
        self.rtype = rtype


def split_units(stmts):
    units, i = [], 0
    while i < len(stmts):
        ln, s = stmts[i]
        m = re.match(r"^MODULE\s+([A-Z_]\w*)$", s)
        hdr = None
        if m:
            hdr = ("module", m.group(1), [], None)
        m = m or None
        if hdr is None:
            m = re.match(r"^PROGRAM\s+([A-Z_]\w*)$", s)
            if m:
                hdr = ("program", m.group(1), [], None)
        if hdr is None:
            m = re.match(r"^SUBROUTINE\s+([A-Z_]\w*)\s*(?:\((.*)\))?$", s)
            if m:
                hdr = ("subroutine", m.group(1), [a.strip() for a in (m.group(2) or "").split(",") if a.strip()], None)
        if hdr is None:
            m = re.match(r"^(DOUBLE\s*PRECISION|INTEGER|REAL|LOGICAL)?\s*FUNCTION\s+([A-Z_]\w*)\s*\((.*)\)$", s)
            if m:
                hdr = ("function", m.group(2), [a.strip() for a in m.group(3).split(",") if a.strip()],
                       _base_type(m.group(1)) if m.group(1) else "r4")
        if hdr is None:
            raise FortranError(f"line {ln}: statement outside a program unit: {s!r}")
        kind, name, args, rtype = hdr
        body, i = [], i + 1
        depth_type = 0
        while i < len(stmts):
            ln2, s2 = stmts[i]
            if re.match(r"^TYPE\s+[A-Z_]\w*$", s2):
                depth_type += 1
            if re.match(r"^END\s*TYPE", s2):
                depth_type -= 1
            if depth_type == 0 and (s2 == "END" or re.match(
                    r"^END\s*(SUBROUTINE|PROGRAM|MODULE|FUNCTION)\b", s2)):
                i += 1
                break
            body.append((ln2, s2))
            i += 1
        units.append(Unit(kind, name, args, body, rtype))
    return units


class Program:
    """Translate and run one Fortran source file."""

    def __init__(self, text, overrides=None, files=None, stubs=(), skip_lines=()):
        self.overrides = {k.upper(): v for k, v in (overrides or {}).items()}
        self.stubs = {s.upper() for s in stubs}
        self.skip_lines = set(skip_lines)
        stmts = [(ln, s) for ln, s in read_statements(text) if ln not in self.skip_lines]
        self.units = {u.name: u for u in split_units(stmts)}
        self.io = _IO(files)
        self.M = type("ModuleVars", (), {})()
        self.msyms = {}      # module symbols
        self.types = {}      # type name -> {comp: Sym}
        self.classes = {}
        self.funcs = {}      # translated subprograms
        self.sigs = {}       # name -> (arg names, arg syms)
        self.env = {"np": np, "math": math, "_f32": _f32, "_idiv": _idiv, "_imod": _imod,
                    "_nint": _nint, "_seqsum": _seqsum, "_r4fn": _r4fn, "_powi": _powi,
                    "_io": self.io, "_MOD": self.M, "_Stop": _Stop, "_aos": _aos, "_aos_set": _aos_set,
                    "_prog": self}
        for u in self.units.values():
            if u.kind == "module":
                self._load_module(u)

    # -- module ---------------------------------------------------------------
    def _load_module(self, u):
        i = 0
        st = u.stmts
        while i < len(st):
            ln, s = st[i]
            m = re.match(r"^TYPE\s+([A-Z_]\w*)$", s)
            if m:
                comps, i = {}, i + 1
                while not re.match(r"^END\s*TYPE", st[i][1]):
                    for sym in self._decl(st[i][1], where="comp"):
                        comps[sym.name] = sym
                    i += 1
                self.types[m.group(1)] = comps
                i += 1
                continue
            if s.startswith("IMPLICIT") or s.startswith("USE "):
                i += 1
                continue
            for sym in self._decl(s, where="module"):
                self.msyms[sym.name] = sym
                self._realize_module_sym(sym)
            i += 1
        for tname, comps in self.types.items():
            for c in comps.values():
                c.lbs = [self._const_int(d[0]) for d in c.dims] if c.dims else None
            self.classes[tname] = self._make_class(tname, comps)

    def _make_class(self, tname, comps):
        prog = self

        class Obj:
            __slots__ = tuple(comps)

            def __init__(self):
                for c in comps.values():
                    if c.dims:
                        shape = [prog._const_int(hi) - prog._const_int(lo) + 1 for lo, hi in c.dims]
                        setattr(self, c.name, np.zeros(shape, dtype=_np_dtype(c.typ)))
                    else:
                        setattr(self, c.name, _zero(c.typ))

        Obj.__name__ = tname
        return Obj

    def _realize_module_sym(self, sym):
        if sym.param:
            v = self._eval_const(sym.init if sym.name not in self.overrides else self.overrides[sym.name],
                                 sym.typ, sym.dims)
            sym.value = v
            setattr(self.M, sym.name, v)
            return
        val = self._new_storage(sym)
        if sym.init is not None:
            init = self.overrides.get(sym.name, sym.init)
            v = self._eval_const(init, sym.typ, sym.dims)
            if isinstance(val, np.ndarray):
                val[...] = v
            else:
                val = v
        setattr(self.M, sym.name, val)

    def _const_int(self, e):
        if isinstance(e, int):
            return e
        return int(self._eval_const(e, "i", None))

    def _eval_const(self, text, typ, dims):
        tr = _Translator(self, {}, "module")
        code, t, arr = tr.expr(parse_expr(text) if isinstance(text, str) else text)
        v = eval(code, self.env)
        if dims:
            shape = [self._const_int(hi) - self._const_int(lo) + 1 for lo, hi in dims]
            a = np.zeros(shape, dtype=_np_dtype(typ))
            a[...] = v
            return a
        return _convert_value(v, typ)

    def _new_storage(self, sym):
        if sym.typ[0] == "t":
            cls = self.classes.get(sym.typ[1])
            if cls is None:
                raise FortranError(f"unknown type {sym.typ[1]}")
            if sym.dims:
                n = self._const_int(sym.dims[0][1]) - self._const_int(sym.dims[0][0]) + 1
                return [cls() for _ in range(n)]
            return cls()
        if sym.dims:
            shape = [self._const_int(hi) - self._const_int(lo) + 1 for lo, hi in sym.dims]
            return np.zeros(shape, dtype=_np_dtype(sym.typ))
        return _zero(sym.typ)

    # -- declarations ---------------------------------------------------------
    def _decl(self, s, where):
        m = _TYPE_KW.match(s)
        if not m:
            raise FortranError(f"not a declaration: {s!r}")
        kw, tname, rest = m.group(1), m.group(2), m.group(3)
        typ = ("t", tname) if tname else _base_type(kw)
        rest = rest.strip()
        attrs = []
        if "::" in rest:
            a, ents = rest.split("::", 1)
            attrs = [x.strip() for x in _split_top(a.lstrip(","))] if a.strip() else []
        else:
            ents = rest
        param = any(x == "PARAMETER" for x in attrs)
        dim_attr = None
        for x in attrs:
            mm = re.match(r"^DIMENSION\s*\((.*)\)$", x)
            if mm:
                dim_attr = _split_top(mm.group(1))
        syms = []
        for e in _split_top(ents):
            name, dims, init = _parse_entity(e)
            dims = dims or dim_attr
            pd = None
            if dims:
                pd = []
                for d in dims:
                    if ":" in d:
                        lo, hi = d.split(":", 1)
                        pd.append((lo.strip() or "1", hi.strip()))
                    else:
                        pd.append(("1", d.strip()))
            syms.append(Sym(name, typ, pd, param=param, where=where, init=init))
        return syms

    # -- subprograms ------------------------------------------------------------
    def sub(self, name):
        name = name.upper()
        if name in self.funcs:
            return self.funcs[name]
        if name in self.stubs:
            fn = lambda *a: a  # noqa: E731
            self.funcs[name] = fn
            return fn
        u = self.units.get(name)
        if u is None:
            raise FortranError(f"no subprogram {name}")
        src = _Translator(self, {}, u.kind, unit=u).translate_unit()
        ns = {}
        try:
            exec(compile(src, f"<fortran {name}>", "exec"), self.env, ns)
        except SyntaxError as e:
            raise FortranError(f"generated code for {name} does not compile: {e}\n{src}")
        fn = ns[f"F_{name}"]
        self.funcs[name] = fn
        self.env[f"F_{name}"] = fn
        return fn

    def run(self):
        main = [u for u in self.units.values() if u.kind == "program"]
        if len(main) != 1:
            raise FortranError("expected one PROGRAM")
        fn = self.sub(main[0].name)
        try:
            frame = fn()
        except _Stop as s:
            frame = s.frame
        return frame


def _np_dtype(typ):
    return {"r8": np.float64, "r4": np.float32, "i": np.int64, "l": np.bool_, "c": object}[typ]


def _zero(typ):
    return {"r8": 0.0, "r4": _f32(0.0), "i": 0, "l": False, "c": ""}[typ]


def _convert_value(v, typ):
    if isinstance(v, np.ndarray):
        return v
    if typ == "r8":
        return float(v)
    if typ == "r4":
        return _f32(v)
    if typ == "i":
        return int(v)
    if typ == "l":
        return bool(v)
    return v


def _aos(objs, comp):
    return np.array([getattr(o, comp) for o in objs])


def _aos_set(objs, comp, value):
    if isinstance(value, np.ndarray) and value.ndim and value.shape[0] == len(objs) and \
            np.ndim(getattr(objs[0], comp)) == value.ndim - 1:
        for o, v in zip(objs, value):
            _set_comp(o, comp, v)
    else:
        for o in objs:
            _set_comp(o, comp, value)


def _set_comp(o, comp, v):
    cur = getattr(o, comp)
    if isinstance(cur, np.ndarray):
        cur[...] = v
    elif isinstance(cur, float):
        setattr(o, comp, float(v))
    elif isinstance(cur, np.float32):
        setattr(o, comp, _f32(v))
    elif isinstance(cur, bool):
        setattr(o, comp, bool(v))
    else:
        setattr(o, comp, int(v))


# ----------------------------------------------------------------------------
# translation of one program unit into a Python function
# ----------------------------------------------------------------------------

_INTRINSIC_RESULT = {"DBLE": "r8", "DFLOAT": "r8", "FLOAT": "r4", "REAL": "r4", "SNGL": "r4",
                     "INT": "i", "NINT": "i", "IDINT": "i"}
_SAME_TYPE = {"SQRT", "DSQRT", "SIN", "DSIN", "COS", "DCOS", "EXP", "DEXP", "ABS", "DABS", "TANH",
              "LOG", "DLOG"}


class _Translator:
    def __init__(self, prog, syms, kind, unit=None):
        self.prog, self.syms, self.kind, self.unit = prog, dict(syms), kind, unit
        self.lines = []
        self.ind = 1
        self.tmp = 0
        self.locals_persist = []

    # -- symbol lookup ----------------------------------------------------------
    def lookup(self, name):
        if name in self.syms:
            return self.syms[name]
        return self.prog.msyms.get(name)

    def ref(self, sym):
        if sym.where == "module":
            return f"_MOD.{sym.name}"
        return sym.name

    def lbs(self, sym):
        if sym.lbs is None:
            sym.lbs = [self.prog._const_int(lo) for lo, _ in sym.dims]
        return sym.lbs

    # -- expressions --------------------------------------------------------------
    def expr(self, e):
        """-> (python code, scalar type, is_array)"""
        k = e[0]
        if k == "num":
            if e[2] == "i":
                return str(e[1]), "i", False
            if e[2] == "r8":
                return repr(float(e[1])), "r8", False
            return f"_f32({e[1]!r})", "r4", False
        if k == "log":
            return ("True" if e[1] else "False"), "l", False
        if k == "str":
            return repr(e[1]), "c", False
        if k == "paren":
            c, t, a = self.expr(e[1])
            return f"({c})", t, a
        if k == "neg":
            c, t, a = self.expr(e[1])
            return f"(-{c})", t, a
        if k == "not":
            c, t, a = self.expr(e[1])
            return (f"np.logical_not({c})" if a else f"(not {c})"), "l", a
        if k == "ctor":
            parts = [self.expr(x) for x in e[1]]
            t = _promote([p[1] for p in parts])
            items = ", ".join(self.conv(c, tt, t) for c, tt, _ in parts)
            return f"np.array([{items}], dtype=np.{_np_dtype(t).__name__})", t, True
        if k == "op":
            return self.binop(e)
        if k in ("name", "ref", "comp"):
            return self.designator(e)
        raise FortranError(f"cannot translate {e!r}")

    def conv(self, code, frm, to):
        if frm == to or to in ("l", "c"):
            return code
        if to == "r8":
            return f"float({code})" if frm in ("r4",) else code
        if to == "r4":
            return f"_f32({code})" if frm == "r8" else code
        return code

    def conv_arr(self, code, frm, to, is_arr):
        if not is_arr:
            return self.conv(code, frm, to)
        if frm == to:
            return code
        return f"np.asarray({code}, dtype=np.{_np_dtype(to).__name__})"

    def binop(self, e):
        _, op, a, b = e
        ca, ta, aa = self.expr(a)
        cb, tb, ab = self.expr(b)
        arr = aa or ab
        if op in (".AND.", ".OR.", ".EQV.", ".NEQV."):
            if arr:
                f = {".AND.": "np.logical_and", ".OR.": "np.logical_or", ".EQV.": "np.equal",
                     ".NEQV.": "np.not_equal"}[op]
                return f"{f}({ca}, {cb})", "l", True
            pyop = {".AND.": "and", ".OR.": "or", ".EQV.": "==", ".NEQV.": "!="}[op]
            return f"({ca} {pyop} {cb})", "l", False
        if op == "**":
            t = _promote([ta, tb]) if tb != "i" else ta
            if b[0] == "num" and b[2] == "i":
                n = b[1]
                if n == 2:
                    return f"({ca}*{ca})" if ca.isidentifier() else f"_powi({ca}, 2)", ta, aa
                return f"_powi({ca}, {n})", ta, aa
            if tb == "i":
                return f"_powi({ca}, {cb})", ta, aa
            ca2, cb2 = self.conv(ca, ta, t), self.conv(cb, tb, t)
            return f"({ca2} ** {cb2})", t, arr
        if op in ("==", "!=", "<", "<=", ">", ">="):
            t = _promote([ta, tb]) if ta in _RANK and tb in _RANK else ta
            ca2 = self.conv_arr(ca, ta, t, aa) if ta in _RANK else ca
            cb2 = self.conv_arr(cb, tb, t, ab) if tb in _RANK else cb
            return f"({ca2} {op} {cb2})", "l", arr
        t = _promote([ta, tb])
        ca2, cb2 = self.conv_arr(ca, ta, t, aa), self.conv_arr(cb, tb, t, ab)
        if op == "/" and t == "i":
            if arr:
                raise FortranError("integer array division is not supported")
            return f"_idiv({ca2}, {cb2})", "i", False
        return f"({ca2} {op} {cb2})", t, arr

    def designator(self, e):
        """names, array elements/sections, components, intrinsic and function calls."""
        if e[0] == "name":
            name = e[1]
            sym = self.lookup(name)
            if sym is None:
                raise FortranError(f"unknown name {name} in {self.unit.name if self.unit else 'module'}")
            if sym.param and sym.value is not None and not isinstance(sym.value, np.ndarray):
                return repr_const(sym.value, sym.typ), sym.typ, False
            t = sym.typ if sym.typ[0] != "t" else sym.typ
            return self.ref(sym), t if isinstance(t, str) else t, bool(sym.dims)
        if e[0] == "ref":
            base, args = e[1], e[2]
            if base[0] == "name":
                name = base[1]
                sym = self.lookup(name)
                if sym is None:
                    return self.call_function(name, args)
                return self.subscript(self.ref(sym), sym, args)
            if base[0] == "comp":
                code, t, isarr, csym = self.component(base)
                return self.subscript(code, csym, args)
            raise FortranError(f"cannot subscript {base!r}")
        if e[0] == "comp":
            code, t, isarr, csym = self.component(e)
            return code, t, isarr
        raise FortranError(repr(e))

    def component(self, e):
        """obj%comp -> (code, type, is_array, component sym)."""
        _, base, cname = e
        if base[0] == "name":
            bsym = self.lookup(base[1])
            if bsym is None or bsym.typ[0] != "t":
                raise FortranError(f"{base[1]} is not a derived-type variable")
            tdef = self.prog.types[bsym.typ[1]]
            csym = tdef[cname]
            if bsym.dims:  # whole array of structures -> array of component values
                return f"_aos({self.ref(bsym)}, {cname!r})", csym.typ, True, csym
            return f"{self.ref(bsym)}.{cname}", csym.typ, bool(csym.dims), csym
        if base[0] == "ref" and base[1][0] == "name":
            bsym = self.lookup(base[1][1])
            if bsym is None or bsym.typ[0] != "t":
                raise FortranError(f"{base[1][1]} is not a derived-type array")
            idx = self.expr(base[2][0])
            lb = self.lbs(bsym)[0]
            tdef = self.prog.types[bsym.typ[1]]
            csym = tdef[cname]
            code = f"{self.ref(bsym)}[{self.offset(idx[0], lb)}].{cname}"
            return code, csym.typ, bool(csym.dims), csym
        raise FortranError(f"unsupported component reference {e!r}")

    def offset(self, code, lb):
        if lb == 0:
            return code
        return f"({code})-{lb}"

    def subscript(self, code, sym, args):
        if not sym.dims:
            raise FortranError(f"{sym.name} is not an array")
        lbs = self.lbs(sym)
        if len(args) != len(lbs):
            raise FortranError(f"rank mismatch for {sym.name}")
        parts, is_arr = [], False
        for a, lb in zip(args, lbs):
            if a[0] == "slice":
                is_arr = True
                lo = "" if a[1] is None else self.offset(self.expr(a[1])[0], lb)
                hi = "" if a[2] is None else f"({self.offset(self.expr(a[2])[0], lb)})+1"
                parts.append(f"{lo}:{hi}")
            else:
                c, t, arr = self.expr(a)
                if t != "i":
                    raise FortranError(f"non-integer subscript of {sym.name}")
                parts.append(self.offset(c, lb))
        return f"{code}[{', '.join(parts)}]", sym.typ, is_arr

    def call_function(self, name, args):
        cargs = [self.expr(a) for a in args]
        if name in _INTRINSIC_RESULT:
            c, t, arr = cargs[0]
            rt = _INTRINSIC_RESULT[name]
            if arr:
                if rt == "i":
                    return f"np.trunc({c}).astype(np.int64)", "i", True
                return f"np.asarray({c}, dtype=np.{_np_dtype(rt).__name__})", rt, True
            if rt == "r8":
                return f"float({c})", "r8", False
            if rt == "r4":
                return f"_f32({c})", "r4", False
            if name == "NINT":
                return f"_nint({c})", "i", False
            return f"int({c})", "i", False
        if name in _SAME_TYPE:
            c, t, arr = cargs[0]
            base = name.lstrip("D") if name not in ("DABS",) else "ABS"
            base = {"SQRT": "sqrt", "SIN": "sin", "COS": "cos", "EXP": "exp", "ABS": "abs",
                    "TANH": "tanh", "LOG": "log", "QRT": "sqrt", "IN": "sin", "OS": "cos",
                    "XP": "exp", "ABS_": "abs", "LOG_": "log"}.get(base, base.lower())
            if name in ("DSQRT",):
                base = "sqrt"
            if name in ("DSIN",):
                base = "sin"
            if name in ("DCOS",):
                base = "cos"
            if name in ("DEXP",):
                base = "exp"
            if name in ("DLOG",):
                base = "log"
            if base == "abs":
                return (f"np.abs({c})" if arr else f"abs({c})"), t, arr
            if arr:
                return f"np.{base}({c})", t, True
            if t == "r4":
                return f"_r4fn('{base}f', {c})", "r4", False
            return f"math.{base}({self.conv(c, t, 'r8')})", "r8", False
        if name in ("MAX", "MIN", "DMAX1", "DMIN1", "AMAX1", "AMIN1"):
            t = _promote([x[1] for x in cargs])
            f = "max" if "MAX" in name else "min"
            return f"{f}({', '.join(self.conv(c, tt, t) for c, tt, _ in cargs)})", t, False
        if name == "MOD":
            (ca, ta, _), (cb, tb, _) = cargs
            t = _promote([ta, tb])
            if t == "i":
                return f"_imod({ca}, {cb})", "i", False
            return f"math.fmod({self.conv(ca, ta, t)}, {self.conv(cb, tb, t)})", t, False
        if name == "SUM":
            c, t, arr = cargs[0]
            return f"_seqsum({c})", t, False
        u = self.prog.units.get(name)
        if u is not None and u.kind == "function":
            self.prog.sub(name)
            return f"F_{name}({', '.join(c for c, _, _ in cargs)})", u.rtype, False
        raise FortranError(f"unknown function or array {name}")

    # -- statements -------------------------------------------------------------
    def emit(self, line):
        self.lines.append("    " * self.ind + line)

    def lvalue(self, e):
        """assignment target -> (code, scalar type, is_array, setter kind, component info)"""
        if e[0] == "name":
            sym = self.lookup(e[1])
            if sym is None:
                raise FortranError(f"assignment to undeclared {e[1]}")
            return self.ref(sym), sym.typ, bool(sym.dims), "var", None
        if e[0] == "ref":
            c, t, arr = self.designator(e)
            return c, t, arr, "elem", None
        if e[0] == "comp":
            base = e[1]
            if base[0] == "name":
                bsym = self.lookup(base[1])
                if bsym is not None and bsym.dims:
                    return f"{self.ref(bsym)}", self.prog.types[bsym.typ[1]][e[2]].typ, True, "aos", e[2]
            c, t, arr, csym = self.component(e)
            return c, t, arr, ("elem" if arr else "comp"), csym
        raise FortranError(f"bad assignment target {e!r}")

    def assign(self, lhs, rhs):
        c, t, arr, kind, extra = self.lvalue(lhs)
        rc, rt, rarr = self.expr(rhs)
        if kind == "aos":
            self.emit(f"_aos_set({c}, {extra!r}, {rc})")
            return
        if arr:
            self.emit(f"{c}[...] = {rc}" if not c.endswith("]") else f"{c} = {rc}")
            return
        if rarr:
            raise FortranError(f"array value assigned to scalar {c}")
        self.emit(f"{c} = {self.conv_assign(rc, rt, t)}")

    def conv_assign(self, code, frm, to):
        if to == "r8":
            return code if frm == "r8" else f"float({code})"
        if to == "r4":
            return code if frm == "r4" else f"_f32({code})"
        if to == "i":
            return code if frm == "i" else f"int({code})"
        if to == "l":
            return code
        return code

    def translate_unit(self):
        u = self.unit
        args = u.args
        decls = []
        body = []
        for ln, s in u.stmts:
            if s.startswith("USE ") or s.startswith("IMPLICIT"):
                continue
            if _looks_like_decl(s):
                decls.append((ln, s))
                continue
            if s.startswith("DATA "):
                raise FortranError(f"line {ln}: DATA is not supported")
            body.append((ln, s))
        for ln, s in decls:
            for sym in self.prog._decl(s, where="local"):
                if sym.name in self.syms and self.syms[sym.name].where == "arg":
                    old = self.syms[sym.name]
                    sym.where = "arg"
                self.syms[sym.name] = sym
        for a in args:
            if a not in self.syms:
                raise FortranError(f"{u.name}: undeclared dummy {a}")
            self.syms[a].where = "arg"
        if u.kind == "function":
            if u.name not in self.syms:
                self.syms[u.name] = Sym(u.name, u.rtype)
        fname = f"F_{u.name}"
        # persistent locals (static storage)
        store = {}
        for s in self.syms.values():
            if s.where == "local":
                if s.param:
                    s.value = self.prog._eval_const(self.prog.overrides.get(s.name, s.init), s.typ, s.dims)
                    store[s.name] = s.value
                    continue
                v = self.prog._new_storage(s)
                if s.init is not None:
                    iv = self.prog._eval_const(s.init, s.typ, s.dims)
                    if isinstance(v, np.ndarray):
                        v[...] = iv
                    else:
                        v = iv
                store[s.name] = v
        self.prog.env[f"_S_{u.name}"] = store
        scal = [n for n, v in store.items() if not isinstance(v, (np.ndarray, list)) and
                not hasattr(v, "__slots__")]
        head = f"def {fname}({', '.join(args)}):"
        self.lines = [head]
        self.ind = 1
        self.emit(f"_S = _S_{u.name}")
        for n in store:
            self.emit(f"{n} = _S[{n!r}]")
        # the value-result tuple for RETURN/end
        self.ret_names = list(args)
        self.save_names = scal
        if u.kind == "function":
            self.ret_expr = u.name
        else:
            self.ret_expr = "(" + "".join(f"{a}, " for a in args) + ")"
        self.block(body, 0, len(body))
        self.emit_return()
        return "\n".join(self.lines) + "\n"

    def emit_return(self):
        for n in self.save_names:
            self.emit(f"_S[{n!r}] = {n}")
        if self.unit.kind == "program":
            self.emit("return locals()")
        else:
            self.emit(f"return {self.ret_expr}")

    def block(self, st, i, end):
        """translate statements st[i:end]"""
        while i < end:
            ln, s = st[i]
            try:
                i = self.statement(st, i, end)
            except FortranError as e:
                raise FortranError(f"line {ln}: {s!r}: {e}") from None

    def _find_end(self, st, i, end, open_re, close_re, mid_re=None):
        depth, mids, j = 0, [], i
        while j < end:
            s = st[j][1]
            if open_re(s):
                depth += 1
            elif close_re(s):
                depth -= 1
                if depth == 0:
                    return j, mids
            elif mid_re and depth == 1 and mid_re(s):
                mids.append(j)
            j += 1
        raise FortranError("unterminated block")

    def statement(self, st, i, end):
        ln, s = st[i]
        # IF ... THEN blocks
        if re.match(r"^IF\s*\(", s):
            p = s.index("(")
            q = _matching_paren(s, p)
            cond = s[p + 1:q]
            rest = s[q + 1:].strip()
            if rest == "THEN":
                j, mids = self._find_end(
                    st, i, end,
                    lambda x: bool(re.match(r"^IF\s*\(", x)) and x.endswith("THEN") and _if_then(x),
                    lambda x: bool(re.match(r"^END\s*IF$", x)),
                    lambda x: bool(re.match(r"^ELSE\s*IF\s*\(", x)) or x == "ELSE")
                cc, ct, _ = self.expr(parse_expr(cond))
                self.emit(f"if {cc}:")
                bounds = [i] + mids + [j]
                for k in range(len(bounds) - 1):
                    a, b = bounds[k], bounds[k + 1]
                    if k > 0:
                        hs = st[a][1]
                        if hs == "ELSE":
                            self.emit("else:")
                        else:
                            p2 = hs.index("(")
                            q2 = _matching_paren(hs, p2)
                            c2, _, _ = self.expr(parse_expr(hs[p2 + 1:q2]))
                            self.emit(f"elif {c2}:")
                    self.ind += 1
                    n0 = len(self.lines)
                    self.block(st, a + 1, b)
                    if len(self.lines) == n0:
                        self.emit("pass")
                    self.ind -= 1
                return j + 1
            # logical IF
            cc, ct, _ = self.expr(parse_expr(cond))
            self.emit(f"if {cc}:")
            self.ind += 1
            self.statement([(ln, rest)], 0, 1)
            self.ind -= 1
            return i + 1
        m = re.match(r"^DO\s+WHILE\s*\((.*)\)$", s)
        if m:
            j, _ = self._find_end(st, i, end, _is_do, _is_enddo)
            cc, _, _ = self.expr(parse_expr(m.group(1)))
            self.emit(f"while {cc}:")
            self.ind += 1
            n0 = len(self.lines)
            self.block(st, i + 1, j)
            if len(self.lines) == n0:
                self.emit("pass")
            self.ind -= 1
            return j + 1
        m = re.match(r"^DO\s+([A-Z_]\w*)\s*=\s*(.*)$", s)
        if m:
            j, _ = self._find_end(st, i, end, _is_do, _is_enddo)
            var = m.group(1)
            parts = _split_top(m.group(2))
            lo = self.expr(parse_expr(parts[0]))[0]
            hi = self.expr(parse_expr(parts[1]))[0]
            step = self.expr(parse_expr(parts[2]))[0] if len(parts) > 2 else "1"
            vsym = self.lookup(var)
            vref = self.ref(vsym)
            stop = f"({hi})+1" if step == "1" else f"({hi})+(1 if ({step})>0 else -1)"
            if vsym.where == "module":
                self.emit(f"for _dv in range({lo}, {stop}, {step}):")
                self.ind += 1
                self.emit(f"{vref} = _dv")
            else:
                self.emit(f"for {vref} in range({lo}, {stop}, {step}):")
                self.ind += 1
            n0 = len(self.lines)
            self.block(st, i + 1, j)
            if len(self.lines) == n0:
                self.emit("pass")
            self.ind -= 1
            return j + 1
        if s in ("EXIT",):
            self.emit("break")
            return i + 1
        if s in ("CYCLE",):
            self.emit("continue")
            return i + 1
        if s in ("CONTINUE",):
            self.emit("pass")
            return i + 1
        if s == "RETURN":
            self.emit_return()
            return i + 1
        if s == "STOP" or s.startswith("STOP "):
            self.emit("raise _Stop(locals())")
            return i + 1
        if s == "PAUSE" or s.startswith("PAUSE "):
            return i + 1
        m = re.match(r"^CALL\s+([A-Z_]\w*)\s*(?:\((.*)\))?$", s)
        if m:
            self.call(m.group(1), _split_top(m.group(2)) if m.group(2) else [])
            return i + 1
        m = re.match(r"^(PRINT\b.*|CLOSE\s*\(.*\))$", s)
        if m:
            return i + 1
        m = re.match(r"^OPEN\s*\((.*)\)$", s)
        if m:
            args = _split_top(m.group(1))
            unit = args[0].replace("UNIT=", "")
            fname = None
            for a in args[1:]:
                mm = re.match(r"^FILE\s*=\s*['\"](.*)['\"]$", a)
                if mm:
                    fname = mm.group(1)
            uc = self.expr(parse_expr(unit))[0]
            self.emit(f"_io.open({uc}, {fname!r})")
            return i + 1
        m = re.match(r"^WRITE\s*\(", s)
        if m:
            p = s.index("(")
            q = _matching_paren(s, p)
            ctl = _split_top(s[p + 1:q])
            items = _split_top(s[q + 1:].strip())
            if ctl[0] == "*":
                return i + 1
            uc = self.expr(parse_expr(ctl[0]))[0]
            vals = [self.expr(parse_expr(x))[0] for x in items]
            self.emit(f"_io.write({uc}, [{', '.join(vals)}])")
            return i + 1
        m = re.match(r"^READ\s*\(", s)
        if m:
            p = s.index("(")
            q = _matching_paren(s, p)
            ctl = _split_top(s[p + 1:q])
            items = _split_top(s[q + 1:].strip())
            uc = self.expr(parse_expr(ctl[0]))[0]
            sizes = []
            targets = []
            for x in items:
                c, t, arr, kind, extra = self.lvalue(parse_expr(x))
                targets.append((c, t, arr, kind, extra))
            self.emit(f"_rd = []")
            for (c, t, arr, kind, extra) in targets:
                if arr:
                    self.emit(f"_n = np.size({c})")
                else:
                    self.emit("_n = 1")
                self.emit("_rd.append(_n)")
            self.emit(f"_vals = _io.read({uc}, sum(_rd))")
            self.emit("_k = 0")
            for idx, (c, t, arr, kind, extra) in enumerate(targets):
                if arr:
                    self.emit(f"{c}[...] = np.array(_vals[_k:_k + _rd[{idx}]]).reshape(np.shape({c}), order='F')"
                              if not c.endswith("]") else
                              f"{c} = np.array(_vals[_k:_k + _rd[{idx}]]).reshape(np.shape({c}), order='F')")
                else:
                    self.emit(f"{c} = {self.conv_assign(f'_vals[_k]', 'r8', t)}")
                self.emit(f"_k += _rd[{idx}]")
            return i + 1
        if s.startswith("CALL CPU_TIME") or re.match(r"^CALL\s+CPU_TIME", s):
            return i + 1
        k = _assign_pos(s)
        if k > 0:
            lhs = parse_expr(s[:k])
            rhs = parse_expr(s[k + 1:])
            self.assign(lhs, rhs)
            return i + 1
        raise FortranError("unsupported statement")

    def call(self, name, arg_texts):
        if name == "CPU_TIME":
            c, t, arr, kind, extra = self.lvalue(parse_expr(arg_texts[0]))
            self.emit(f"{c} = {self.conv_assign('0.0', 'r8', t)}")
            return
        if name in self.prog.stubs:
            return
        u = self.prog.units.get(name)
        if u is None:
            raise FortranError(f"CALL of unknown subroutine {name}")
        self.prog.sub(name)  # translate callee first (its dummy types)
        callee_syms = self.prog._dummy_syms(name)
        args = [parse_expr(a) for a in arg_texts]
        codes = []
        backs = []
        for k, a in enumerate(args):
            dsym = callee_syms[k]
            if dsym.dims or dsym.typ[0] == "t":
                c, t, arr = self.expr(a) if a[0] != "comp" else self.designator(a)
                codes.append(c)
            else:
                c, t, arr = self.expr(a)
                codes.append(self.conv(c, t, dsym.typ) if t in _RANK and dsym.typ in _RANK else c)
                if a[0] in ("name", "ref", "comp"):
                    try:
                        lc, lt, larr, lkind, _ = self.lvalue(a)
                    except FortranError:
                        continue
                    if not larr and lkind != "aos":
                        sym = self.lookup(a[1]) if a[0] == "name" else None
                        if sym is not None and sym.param:
                            continue
                        backs.append((k, lc, lt, dsym.typ))
        self.emit(f"_r = F_{name}({', '.join(codes)})")
        for k, lc, lt, dt in backs:
            self.emit(f"{lc} = {self.conv_assign(f'_r[{k}]', dt, lt)}")


def _if_then(s):
    p = s.index("(")
    q = _matching_paren(s, p)
    return s[q + 1:].strip() == "THEN"


def _is_do(s):
    return bool(re.match(r"^DO(\s+WHILE\s*\(|\s+[A-Z_]\w*\s*=|$)", s))


def _is_enddo(s):
    return bool(re.match(r"^END\s*DO$", s))


def _looks_like_decl(s):
    # a declaration, not an assignment whose target starts like a type keyword
    m = _TYPE_KW.match(s)
    if not m:
        return False
    rest = m.group(3).strip()
    if rest.startswith("=") or (rest.startswith("(") and not m.group(2) and _assign_pos(s) >= 0
                                and "::" not in s and not re.match(r"^(CHARACTER)", s)):
        return False
    return True


def _promote(types):
    nums = [t for t in types if t in _RANK]
    if not nums:
        return types[0]
    return max(nums, key=lambda t: _RANK[t])


def repr_const(v, typ):
    if typ == "r4":
        return f"_f32({float(v)!r})"
    if typ == "r8":
        return repr(float(v))
    if typ == "l":
        return "True" if v else "False"
    return repr(int(v))


def _dummy_syms(self, name):
    u = self.units[name]
    if name not in self.sigs:
        tr = _Translator(self, {}, u.kind, unit=u)
        syms = {}
        for ln, s in u.stmts:
            if s.startswith("USE ") or s.startswith("IMPLICIT"):
                continue
            if _looks_like_decl(s):
                for sym in self._decl(s, where="local"):
                    syms[sym.name] = sym
        self.sigs[name] = [syms[a] for a in u.args]
    return self.sigs[name]


Program._dummy_syms = _dummy_syms


def run_program(text, overrides=None, files=None, stubs=(), skip_lines=()):
    """Translate and run a program; returns (main program's variables, I/O
    records per unit, Program)."""
    prog = Program(text, overrides=overrides, files=files, stubs=stubs, skip_lines=skip_lines)
    frame = prog.run()
    return frame, prog.io.written, prog
