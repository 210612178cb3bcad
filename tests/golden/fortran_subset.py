"""TEST INFRASTRUCTURE ONLY: executes Fortran 90 source text of the reference.

A small interpreter for the subset of Fortran that the particle-path
routines of the reference are written in (src/pcl2field/psolve2.F90,
psolve1.F90, charge.F90, src/field/grdcrt.F90, src/field/rhoupd.F90): free
form with `&` continuations, subroutines and functions with `contains`,
`block` constructs, DO loops with optional construct labels, IF blocks and
one-line IFs, CYCLE/EXIT/RETURN, assignments to array elements, sections and
derived-type components, CALLs, and expressions with Fortran precedence and
types.  Integer arithmetic truncates toward zero, mixed arithmetic promotes
to REAL(8), assignments convert to the declared type of the target, and every
REAL(8) operation is one IEEE binary64 operation in left-to-right order
(Python floats), i.e. the reference evaluated without fused multiply-adds.

It is used only by make_golden.py to produce golden fixtures; nothing in the
product or the test run imports it.
"""
from __future__ import annotations

import math
import re

import numpy as np


class FortranError(Exception):
    pass


# ---------------------------------------------------------------- values
class FArray:
    """A Fortran array: numpy data (first index = first dimension) and lower
    bounds.  Sections are numpy views, so writes reach the parent."""

    def __init__(self, data: np.ndarray, lbounds=None):
        self.data = data
        self.lb = list(lbounds) if lbounds is not None else [1] * data.ndim

    def _key(self, idx):
        key = []
        for d, v in enumerate(idx):
            if isinstance(v, slice):
                start = None if v.start is None else v.start - self.lb[d]
                stop = None if v.stop is None else v.stop - self.lb[d] + 1
                key.append(slice(start, stop))
            else:
                key.append(int(v) - self.lb[d])
        return tuple(key)

    def get(self, idx):
        k = self._key(idx)
        r = self.data[k]
        if any(isinstance(v, slice) for v in idx):
            return FArray(r, [1] * r.ndim)
        return r

    def set(self, idx, value):
        k = self._key(idx)
        if isinstance(value, FArray):
            value = value.data
        self.data[k] = value


class DerivedObj:
    """A scalar of a derived type (attributes hold the components)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def is_int(v):
    return isinstance(v, (int, np.integer)) and not isinstance(v, (bool, np.bool_))


def to_real(v):
    return float(v)


def fdiv(a, b):
    if is_int(a) and is_int(b):
        q = abs(int(a)) // abs(int(b))
        return q if (a >= 0) == (b >= 0) else -q
    return float(a) / float(b)


def binop(op, a, b):
    if isinstance(a, FArray) or isinstance(b, FArray):
        # elementwise REAL(8) arithmetic of sections and scalars
        x = a.data if isinstance(a, FArray) else a
        y = b.data if isinstance(b, FArray) else b
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        r = {"+": np.add, "-": np.subtract, "*": np.multiply, "/": np.divide}[op](x, y)
        return FArray(np.asarray(r), [1] * np.ndim(r))
    if op in ("+", "-", "*", "/", "**"):
        if is_int(a) and is_int(b):
            a, b = int(a), int(b)
            if op == "+": return a + b
            if op == "-": return a - b
            if op == "*": return a * b
            if op == "/": return fdiv(a, b)
            return a ** b if b >= 0 else fdiv(1, a ** -b)
        if op == "**" and is_int(b) and 0 <= int(b) <= 4:
            # a real base to a small integer power is multiplied out, as
            # gfortran does: x**2 = x*x, x**3 = (x*x)*x, x**4 = (x*x)*(x*x)
            a, n = float(a), int(b)
            return [1.0, a, a * a, (a * a) * a, (a * a) * (a * a)][n]
        a, b = float(a), float(b)
        if op == "+": return a + b
        if op == "-": return a - b
        if op == "*": return a * b
        if op == "/": return a / b
        return a ** b
    if op in ("==", "/=", "<", "<=", ">", ">="):
        if not (is_int(a) and is_int(b)):
            a, b = float(a), float(b) if not isinstance(b, str) else b
        return {"==": a == b, "/=": a != b, "<": a < b, "<=": a <= b, ">": a > b, ">=": a >= b}[op]
    if op == "//": return str(a) + str(b)
    if op == ".and.": return bool(a) and bool(b)
    if op == ".or.": return bool(a) or bool(b)
    if op == ".eqv.": return bool(a) == bool(b)
    if op == ".neqv.": return bool(a) != bool(b)
    raise FortranError(f"operator {op}")


# ---------------------------------------------------------------- lexer
DOTOPS = {".and.", ".or.", ".not.", ".eq.", ".ne.", ".lt.", ".le.", ".gt.", ".ge.", ".true.", ".false.", ".eqv.",
          ".neqv."}
DOTMAP = {".eq.": "==", ".ne.": "/=", ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">="}
NUM = re.compile(r"(\d+\.\d*|\.\d+|\d+)([de][+-]?\d+)?(_\w+)?")


def tokenize(s: str):
    toks = []
    i = 0
    n = len(s)
    while i < n:
        c = s[i]
        if c.isspace():
            i += 1
            continue
        if c == ".":
            m = re.match(r"\.[a-z]+\.", s[i:])
            if m and m.group(0) in DOTOPS:
                w = m.group(0)
                toks.append(("op", DOTMAP.get(w, w)))
                i += len(w)
                continue
        if c.isdigit() or (c == "." and i + 1 < n and s[i + 1].isdigit()):
            m = NUM.match(s, i)
            txt = m.group(0)
            # "1.eq.2": a trailing '.' that starts a dot operator belongs to it
            if txt.endswith(".") and re.match(r"\.[a-z]+\.", s[m.end() - 1:]) and \
                    re.match(r"\.[a-z]+\.", s[m.end() - 1:]).group(0) in DOTOPS:
                txt = txt[:-1]
            i += len(txt)
            body = re.sub(r"_\w+$", "", txt)
            if re.fullmatch(r"\d+", body):
                toks.append(("num", int(body)))
            elif "d" in body or body != txt:
                toks.append(("num", float(body.replace("d", "e"))))  # double precision (d exponent or kind)
            else:
                toks.append(("num", float(np.float32(float(body)))))  # default real: single precision
            continue
        if c.isalpha() or c == "_":
            m = re.match(r"[a-z_][a-z0-9_]*", s[i:])
            toks.append(("name", m.group(0)))
            i += len(m.group(0))
            continue
        if c == "'" or c == '"':
            j = s.index(c, i + 1)
            toks.append(("str", s[i + 1:j]))
            i = j + 1
            continue
        two = s[i:i + 2]
        if two == "(/" or two == "/)":  # array constructor (/ ... /)
            toks.append(("op", "[" if two == "(/" else "]"))
            i += 2
            continue
        if two in ("**", "==", "/=", "<=", ">=", "=>", "//"):
            toks.append(("op", two))
            i += 2
            continue
        if c in "+-*/()<>,:%=[]":
            toks.append(("op", c))
            i += 1
            continue
        raise FortranError(f"cannot lex {s[i:]!r}")
    return toks


# ---------------------------------------------------------------- expressions
PREC = [(".eqv.", ".neqv."), (".or.",), (".and.",), (".not.",), ("==", "/=", "<", "<=", ">", ">="), ("//",),
        ("+", "-"), ("*", "/"), ("**",)]


class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k] if self.i + k < len(self.t) else (None, None)

    def take(self, kind=None, val=None):
        tok = self.peek()
        if (kind and tok[0] != kind) or (val is not None and tok[1] != val):
            raise FortranError(f"expected {kind} {val}, got {tok}")
        self.i += 1
        return tok

    def at(self, val):
        return self.peek()[1] == val and self.peek()[0] in ("op",)

    def expr(self, level=0):
        if level == len(PREC):
            return self.primary()
        ops = PREC[level]
        if ops == (".not.",):
            if self.at(".not."):
                self.take()
                return ("not", self.expr(level))
            return self.expr(level + 1)
        if ops == ("+", "-"):
            if self.at("-") or self.at("+"):
                op = self.take()[1]
                left = self.expr(level + 1)
                left = ("neg", left) if op == "-" else left
            else:
                left = self.expr(level + 1)
            while self.peek()[0] == "op" and self.peek()[1] in ops:
                op = self.take()[1]
                left = ("bin", op, left, self.expr(level + 1))
            return left
        if ops == ("**",):
            left = self.expr(level + 1)
            if self.at("**"):
                self.take()
                right = self.expr(level)  # right associative
                return ("bin", "**", left, right)
            return left
        left = self.expr(level + 1)
        while self.peek()[0] == "op" and self.peek()[1] in ops:
            op = self.take()[1]
            left = ("bin", op, left, self.expr(level + 1))
        return left

    def primary(self):
        kind, val = self.peek()
        if kind == "num":
            self.take()
            return ("num", val)
        if kind == "str":
            self.take()
            return ("str", val)
        if kind == "op" and val in (".true.", ".false."):
            self.take()
            return ("num", val == ".true.")
        if kind == "op" and val == "(":
            self.take()
            e = self.expr()
            self.take("op", ")")
            return e
        if kind == "op" and val == "[":
            self.take()
            items = [self.expr()]
            while self.at(","):
                self.take()
                items.append(self.expr())
            self.take("op", "]")
            return ("ctor", items)
        if kind == "op" and (val == "-" or val == "+"):
            self.take()
            e = self.primary()
            return ("neg", e) if val == "-" else e
        if kind == "name":
            return self.designator()
        raise FortranError(f"unexpected {kind} {val}")

    def designator(self):
        parts = []
        name = self.take("name")[1]
        args = self.arglist() if self.at("(") else None
        parts.append((name, args))
        while self.at("%"):
            self.take()
            comp = self.take("name")[1]
            a2 = self.arglist() if self.at("(") else None
            parts.append((comp, a2))
        return ("des", parts)

    def arglist(self):
        self.take("op", "(")
        args = []
        if self.at(")"):
            self.take()
            return args
        while True:
            args.append(self.subscript())
            if self.at(","):
                self.take()
                continue
            self.take("op", ")")
            return args

    def subscript(self):
        # keyword argument name=value
        if self.peek()[0] == "name" and self.peek(1) == ("op", "="):
            kw = self.take()[1]
            self.take()
            return ("kw", kw, self.expr())
        lo = hi = None
        if not self.at(":"):
            lo = self.expr()
            if not self.at(":"):
                return lo
        self.take("op", ":")
        if not (self.at(",") or self.at(")")):
            hi = self.expr()
        return ("range", lo, hi)


def parse_expr(s: str):
    p = Parser(tokenize(s))
    e = p.expr()
    if p.i != len(p.t):
        raise FortranError(f"trailing tokens in {s!r}")
    return e


# ---------------------------------------------------------------- source
def clean_lines(text: str):
    out = []
    buf = ""
    for raw in text.splitlines():
        line = raw.rstrip()
        if line.lstrip().startswith("#"):
            continue
        # strip comments (no '!' inside strings in these files)
        q = None
        cut = len(line)
        for i, ch in enumerate(line):
            if q:
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
            elif ch == "!":
                cut = i
                break
        line = line[:cut].rstrip()
        s = line.strip()
        if not s:
            continue
        if buf:
            if s.startswith("&"):
                s = s[1:]
            buf += " " + s
        else:
            buf = s
        if buf.endswith("&"):
            buf = buf[:-1]
            continue
        for part in buf.split(";"):  # no ';' inside strings in these files
            if part.strip():
                out.append(part.strip().lower())
        buf = ""
    return out


class Unit:
    def __init__(self, kind, name, args, result=None):
        self.kind, self.name, self.args, self.result = kind, name, args, result
        self.decls = []      # (type, name, dims or None, init, is_parameter)
        self.body = []
        self.contains = {}


DECL_TYPES = ("integer", "real", "double precision", "logical", "type(", "type (", "character")
HEADER = re.compile(r"^(?:pure\s+|elemental\s+|recursive\s+)*(subroutine|function)\s+(\w+)\s*(?:\(([^)]*)\))?\s*"
                    r"(?:result\s*\((\w+)\))?$")
END_UNIT = re.compile(r"^end(\s*(subroutine|function)\b.*)?$")


def _matching_paren(ln, start):
    depth = 0
    for k in range(start, len(ln)):
        if ln[k] == "(":
            depth += 1
        elif ln[k] == ")":
            depth -= 1
            if depth == 0:
                return k
    raise FortranError(f"unbalanced parentheses: {ln}")


def _split_top(s, sep=","):
    depth, cur, items = 0, "", []
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            items.append(cur)
            cur = ""
        else:
            cur += ch
    items.append(cur)
    return items


def _parse_decl(ln):
    tpart, names = ln.split("::", 1)
    tpart = tpart.strip()
    if tpart.startswith("integer"):
        ty = "integer"
    elif tpart.startswith("logical"):
        ty = "logical"
    elif tpart.startswith("real") or tpart.startswith("double"):
        ty = "real"
    elif tpart.startswith("type"):
        ty = "type:" + re.search(r"type\s*\((\w+)\)", tpart).group(1)
    else:
        ty = "other"
    is_param = "parameter" in tpart
    out = []
    for it in _split_top(names):
        it = it.strip()
        init = None
        eq = [k for k, ch in enumerate(it) if ch == "=" and it[k + 1:k + 2] != "=" and it[k - 1:k] not in "<>/="]
        if eq:
            init = parse_expr(it[eq[0] + 1:].strip())
            it = it[:eq[0]].strip()
        m = re.match(r"^(\w+)\s*(\((.*)\))?$", it)
        dims = Parser(tokenize("(" + m.group(3) + ")")).arglist() if m.group(3) else None
        out.append((ty, m.group(1), dims, init, is_param))
    return out


class SourceParser:
    def __init__(self, lines):
        self.lines = lines
        self.i = 0

    def units(self):
        out = {}
        while self.i < len(self.lines):
            if HEADER.match(self.lines[self.i]):
                u = self.unit()
                out[u.name] = u
            else:
                self.i += 1
        return out

    def unit(self):
        m = HEADER.match(self.lines[self.i])
        u = Unit(m.group(1), m.group(2), [a.strip() for a in (m.group(3) or "").split(",") if a.strip()], m.group(4))
        self.i += 1
        stmts = self.block(lambda l: l == "contains" or END_UNIT.match(l) is not None)
        for st in stmts:
            if st[0] == "decl":
                u.decls.extend(st[1])
            elif st[0] != "nop":
                u.body.append(st)
        if self.lines[self.i] == "contains":
            self.i += 1
            while not END_UNIT.match(self.lines[self.i]):
                if HEADER.match(self.lines[self.i]):
                    sub = self.unit()
                    u.contains[sub.name] = sub
                else:
                    self.i += 1
        self.i += 1  # the END line
        return u

    def block(self, end_pred):
        out = []
        while not end_pred(self.lines[self.i]):
            out.append(self.stmt())
        return out

    def stmt(self):
        ln = self.lines[self.i]
        self.i += 1
        return self.stmt_text(ln)

    def stmt_text(self, ln):
        m = re.match(r"^(\d+)\s+(.*)$", ln)
        if m:  # numeric statement label (the target of a GO TO)
            return ("label", int(m.group(1)), self.stmt_text(m.group(2)))
        if ln == "continue":
            return ("nop",)
        m = re.match(r"^go\s*to\s+(\d+)$", ln)
        if m:
            return ("goto", int(m.group(1)))
        if re.match(r"^(print|write)\b", ln):
            return ("nop",)  # output statements change no value
        label = None
        m = re.match(r"^(\w+)\s*:\s*(do\b.*)$", ln)
        if m:
            label, ln = m.group(1), m.group(2)
        m = re.match(r"^do\s+while\s*\((.*)\)$", ln)
        if m:
            cond = parse_expr(m.group(1))
            body = self.block(lambda l: re.match(r"^end\s*do\b", l) is not None)
            self.i += 1
            return ("dowhile", label, cond, body)
        if re.match(r"^do\b", ln):
            m = re.match(r"^do\s+(\w+)\s*=\s*(.+)$", ln)
            if not m:
                raise FortranError(f"unsupported do: {ln}")
            p = Parser(tokenize(m.group(2)))
            lo = p.expr()
            p.take("op", ",")
            hi = p.expr()
            step = None
            if p.at(","):
                p.take()
                step = p.expr()
            body = self.block(lambda l: re.match(r"^end\s*do\b", l) is not None)
            self.i += 1
            return ("do", label, m.group(1), lo, hi, step, body)
        if re.match(r"^if\s*\(", ln):
            k = _matching_paren(ln, ln.index("("))
            cond = parse_expr(ln[ln.index("(") + 1:k])
            rest = ln[k + 1:].strip()
            if rest != "then":
                return ("if", [(cond, [self.stmt_text(rest)])])
            branches = []
            cur = cond
            while True:
                body = self.block(lambda l: re.match(r"^(else\b|end\s*if\b)", l) is not None)
                branches.append((cur, body))
                ln2 = self.lines[self.i]
                self.i += 1
                if re.match(r"^end\s*if\b", ln2):
                    return ("if", branches)
                m2 = re.match(r"^else\s*if\s*\((.*)\)\s*then$", ln2)
                cur = parse_expr(m2.group(1)) if m2 else None
        if re.match(r"^type\s+\w+$", ln):  # derived-type definition: components are dynamic here
            while not re.match(r"^end\s*type\b", self.lines[self.i]):
                self.i += 1
            self.i += 1
            return ("nop",)
        if ln == "block":
            body = self.block(lambda l: re.match(r"^end\s*block\b", l) is not None)
            self.i += 1
            decls = [d for s_ in body if s_[0] == "decl" for d in s_[1]]
            return ("block", decls, [s_ for s_ in body if s_[0] not in ("decl", "nop")])
        if re.match(r"^cycle\b", ln):
            w = ln.split()
            return ("cycle", w[1] if len(w) > 1 else None)
        if re.match(r"^exit\b", ln):
            w = ln.split()
            return ("exit", w[1] if len(w) > 1 else None)
        if ln == "return":
            return ("return",)
        if re.match(r"^call\b", ln):
            return ("call", parse_expr(ln[4:].strip()))
        if re.match(r"^(use|implicit|include|save|intent)\b", ln):
            return ("nop",)
        if any(ln.startswith(t) for t in DECL_TYPES) and "::" in ln:
            return ("decl", _parse_decl(ln))
        depth = 0
        for k, ch in enumerate(ln):
            if ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
            elif ch == "=" and depth == 0 and ln[k + 1:k + 2] != "=" and ln[k - 1:k] not in "<>/=":
                return ("assign", parse_expr(ln[:k]), parse_expr(ln[k + 1:]))
        raise FortranError(f"unsupported statement: {ln}")


def parse_source(text: str) -> dict:
    return SourceParser(clean_lines(text)).units()


# ---------------------------------------------------------------- execution
class _Cycle(Exception):
    def __init__(self, label):
        self.label = label


class _Exit(Exception):
    def __init__(self, label):
        self.label = label


class _Return(Exception):
    pass


class _Goto(Exception):
    def __init__(self, label):
        self.label = label


class Frame:
    def __init__(self, interp, unit, parent=None):
        self.interp = interp
        self.unit = unit
        self.vars = {}
        self.types = {}
        self.parent = parent  # host scope for contained procedures
        self.absent = set()   # optional dummy arguments not given

    def lookup(self, name):
        f = self
        while f is not None:
            if name in f.vars:
                return f
            f = f.parent
        if name in self.interp.globals:
            return None
        raise FortranError(f"unknown name {name}")


def _libm_tgamma(x):
    """GAMMA: the C library's tgamma (what gfortran calls; Python's
    math.gamma is a different implementation)."""
    import ctypes
    import ctypes.util
    f = ctypes.CDLL(ctypes.util.find_library("m")).tgamma
    f.restype, f.argtypes = ctypes.c_double, [ctypes.c_double]
    return f(float(x))


INTRINSICS = {
    "int": lambda x, *kind: int(x),  # truncation toward zero; the kind argument changes no value here
    "floor": lambda x: int(math.floor(x)),
    "nint": lambda x: int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5)),  # half away from 0
    "dble": float, "real": lambda x, *k: float(x),
    "abs": abs, "sqrt": math.sqrt, "exp": math.exp, "cos": math.cos, "sin": math.sin,
    "dabs": abs, "dsqrt": math.sqrt, "dexp": math.exp, "dcos": math.cos, "dsin": math.sin,
    "log": math.log, "dlog": math.log, "erf": math.erf,  # math.erf is the C library's erf
    "gamma": lambda x: _libm_tgamma(x),
    "mod": lambda a, b: (a - int(a / b) * b) if not (is_int(a) and is_int(b)) else int(math.fmod(a, b)),
}


def fmax(*xs):
    if all(is_int(x) for x in xs):
        return max(int(x) for x in xs)
    r = float(xs[0])
    for x in xs[1:]:
        r = max(r, float(x))
    return r


def fmin(*xs):
    if all(is_int(x) for x in xs):
        return min(int(x) for x in xs)
    r = float(xs[0])
    for x in xs[1:]:
        r = min(r, float(x))
    return r


class Interpreter:
    def __init__(self, units: dict, globals_: dict, externals: dict | None = None, types: dict | None = None):
        self.units = units
        self.globals = globals_
        self.gtypes = types or {}
        self.externals = externals or {}

    # -- calls
    def call(self, name, args, frame=None, kw=None):
        unit = None
        if frame is not None:
            f = frame
            while f is not None and unit is None:
                unit = f.unit.contains.get(name)
                f = f.parent
        if unit is None:
            unit = self.units.get(name)
        if unit is None:
            if name in self.externals:
                return self.externals[name](*args, **(kw or {}))
            raise FortranError(f"unknown procedure {name}")
        host = None
        if frame is not None and name not in self.units:
            # contained procedure: host association with the caller's host unit
            host = frame
            while host.parent is not None and name not in host.unit.contains:
                host = host.parent
        fr = Frame(self, unit, parent=host)
        for (ty, nm, dims, init, is_param) in unit.decls:
            fr.types[nm] = ty
        for a, v in zip(unit.args, args):
            fr.vars[a] = v
        for a, v in (kw or {}).items():
            if a not in unit.args:
                raise FortranError(f"{name}: no dummy argument {a}")
            fr.vars[a] = v
        # dummies not given: absent optional arguments (present() is false)
        fr.absent = {a for a in unit.args if a not in fr.vars}
        for (ty, nm, dims, init, is_param) in unit.decls:
            if nm in fr.absent:
                continue
            if nm in fr.vars:
                if dims is not None and isinstance(fr.vars[nm], FArray):
                    # explicit-shape dummy: rebind bounds
                    lbs = []
                    for d in dims:
                        if d[0] == "range":
                            lbs.append(self.eval(d[1], fr) if d[1] is not None else 1)
                        else:
                            lbs.append(1)
                    fr.vars[nm] = FArray(fr.vars[nm].data, lbs)
                continue
            fr.vars[nm] = self.alloc(ty, dims, init, fr)
        if unit.result:
            fr.vars.setdefault(unit.result, self.alloc(fr.types.get(unit.result, "real"), None, None, fr))
        try:
            self.run_block(unit.body, fr)
        except _Return:
            pass
        self.last_frame = fr
        if unit.kind == "function":
            return fr.vars[unit.result or unit.name]
        return None

    def alloc(self, ty, dims, init, fr):
        if dims is None:
            if init is not None:
                return self.convert(ty, self.eval(init, fr))
            if ty == "integer":
                return 0
            if ty == "logical":
                return False
            if ty.startswith("type:"):
                return DerivedObj()
            return 0.0
        lbs, shape = [], []
        for d in dims:
            if d[0] == "range":
                lo = self.eval(d[1], fr) if d[1] is not None else 1
                hi = self.eval(d[2], fr)
            else:
                lo, hi = 1, self.eval(d, fr)
            lbs.append(int(lo))
            shape.append(int(hi) - int(lo) + 1)
        dt = np.int64 if ty == "integer" else (np.bool_ if ty == "logical" else np.float64)
        return FArray(np.zeros(shape, dtype=dt), lbs)

    def convert(self, ty, v):
        if ty == "integer":
            return int(v) if not is_int(v) else int(v)
        if ty == "real":
            return float(v)
        if ty == "logical":
            return bool(v)
        return v

    # -- statements
    def run_block(self, stmts, fr):
        i = 0
        while i < len(stmts):
            try:
                self.exec(stmts[i], fr)
                i += 1
            except _Goto as g:
                # a GO TO resumes at the labelled statement of this block, or
                # leaves the block for an enclosing one
                for j, st in enumerate(stmts):
                    if st[0] == "label" and st[1] == g.label:
                        i = j
                        break
                else:
                    raise

    def exec(self, st, fr):
        k = st[0]
        if k == "assign":
            self.assign(st[1], self.eval(st[2], fr), fr)
        elif k == "if":
            for cond, body in st[1]:
                if cond is None or self.eval(cond, fr):
                    self.run_block(body, fr)
                    break
        elif k == "do":
            _, label, var, lo, hi, step, body = st
            lo, hi = self.eval(lo, fr), self.eval(hi, fr)
            step = self.eval(step, fr) if step is not None else 1
            n_iter = max(0, (hi - lo + step) // step)
            v = lo
            for _ in range(int(n_iter)):
                self.assign(("des", [(var, None)]), v, fr)
                try:
                    self.run_block(body, fr)
                except _Cycle as c:
                    if c.label not in (None, label):
                        raise
                except _Exit as e:
                    if e.label not in (None, label):
                        raise
                    break
                v += step
            self.assign(("des", [(var, None)]), v, fr)
        elif k == "dowhile":
            _, label, cond, body = st
            while self.eval(cond, fr):
                try:
                    self.run_block(body, fr)
                except _Cycle as c:
                    if c.label not in (None, label):
                        raise
                except _Exit as e:
                    if e.label not in (None, label):
                        raise
                    break
        elif k == "block":
            inner = Frame(self, Unit("block", "block", []), parent=fr)
            for (ty, nm, dims, init, is_param) in st[1]:
                inner.types[nm] = ty
                inner.vars[nm] = self.alloc(ty, dims, init, inner)
            inner.unit.contains = {}
            self.run_block(st[2], inner)
        elif k == "cycle":
            raise _Cycle(st[1])
        elif k == "exit":
            raise _Exit(st[1])
        elif k == "return":
            raise _Return()
        elif k == "call":
            self.do_call(st[1], fr)
        elif k == "nop":
            pass
        elif k == "label":
            self.exec(st[2], fr)
        elif k == "goto":
            raise _Goto(st[1])
        elif k == "decl":
            pass
        else:
            raise FortranError(f"statement {k}")

    def do_call(self, des, fr):
        parts = des[1]
        if len(parts) == 1:
            name, args = parts[0]
            pos = [a for a in (args or []) if not (isinstance(a, tuple) and a[0] == "kw")]
            vals = [self.eval(a, fr) for a in pos]
            # an element of a 1-D array given for an array dummy: sequence
            # association, the dummy starts at that element
            unit = self.units.get(name)
            if unit is not None:
                arr_dummies = {nm for (ty, nm, dims, init, is_param) in unit.decls if dims is not None}
                for q, (a, dummy) in enumerate(zip(pos, unit.args)):
                    if dummy not in arr_dummies or not (isinstance(a, tuple) and a[0] == "des"):
                        continue
                    parts = a[1]
                    if len(parts) != 1 or parts[0][1] is None or len(parts[0][1]) != 1:
                        continue
                    scope, nm, ty = self.resolve(parts[0][0], fr)
                    arr = scope[nm] if scope is not None else None
                    sub = parts[0][1][0]
                    if isinstance(arr, FArray) and arr.data.ndim == 1 and not (isinstance(sub, tuple) and
                                                                              sub[0] == "range"):
                        k0 = int(self.eval(sub, fr)) - arr.lb[0]
                        vals[q] = FArray(arr.data[k0:], [1])
            kw = {a[1]: self.eval(a[2], fr) for a in (args or []) if isinstance(a, tuple) and a[0] == "kw"}
            self.last_frame = None
            self.call(name, vals, fr, kw)
            callee = self.last_frame
            # arguments pass by reference: a scalar variable or component
            # given to an interpreted subroutine gets the dummy's final value
            if callee is not None and callee.unit.name == name:
                for a, v, dummy in zip(pos, vals, callee.unit.args):
                    if isinstance(a, tuple) and a[0] == "des" and not isinstance(v, (FArray, np.ndarray, DerivedObj)):
                        nv = callee.vars.get(dummy, v)
                        if nv is not v:
                            self.assign(a, nv, fr)
            return
        # obj%method(args): type-bound call
        obj = self.eval(("des", parts[:-1]), fr)
        name, args = parts[-1]
        vals = [self.eval_arg(a, fr) for a in (args or [])]
        getattr(obj, name)(*vals)

    def eval_arg(self, a, fr):
        if isinstance(a, tuple) and a[0] == "kw":
            return self.eval(a[2], fr)
        return self.eval(a, fr)

    # -- designators
    def resolve(self, name, fr):
        f = fr
        while f is not None:
            if name in f.vars:
                return f.vars, name, f.types.get(name)
            f = f.parent
        if name in self.globals:
            return self.globals, name, self.gtypes.get(name)
        return None, name, None

    def subs(self, args, fr):
        out = []
        for a in args:
            if isinstance(a, tuple) and a[0] == "range":
                lo = self.eval(a[1], fr) if a[1] is not None else None
                hi = self.eval(a[2], fr) if a[2] is not None else None
                out.append(slice(lo, hi))
            else:
                out.append(self.eval(a, fr))
        return out

    def eval(self, e, fr):
        k = e[0]
        if k == "num":
            return e[1]
        if k == "str":
            return e[1]
        if k == "neg":
            v = self.eval(e[1], fr)
            return FArray(-v.data, v.lb) if isinstance(v, FArray) else -v
        if k == "not":
            return not self.eval(e[1], fr)
        if k == "bin":
            op = e[1]
            a = self.eval(e[2], fr)
            if op == ".and." and not a:
                return False  # Fortran may short-circuit; the routines are side-effect free here
            if op == ".or." and a:
                return True
            return binop(op, a, self.eval(e[3], fr))
        if k == "ctor":
            return [self.eval(x, fr) for x in e[1]]
        if k == "des":
            return self.eval_des(e[1], fr)
        raise FortranError(f"expr {k}")

    def eval_des(self, parts, fr):
        name, args = parts[0]
        scope, nm, ty = self.resolve(name, fr)
        if scope is None and name == "present":
            return args[0][1][0][0] not in fr.absent
        if scope is None:
            # function / intrinsic
            vals = [self.eval_arg(a, fr) for a in (args or [])]
            if name == "max":
                return fmax(*vals)
            if name == "min":
                return fmin(*vals)
            if name in INTRINSICS:
                return INTRINSICS[name](*vals)
            return self.call(name, vals, fr)
        obj = scope[nm]
        if args is not None:
            obj = obj.get(self.subs(args, fr)) if isinstance(obj, FArray) else obj[tuple(self.subs(args, fr))]
        for comp, cargs in parts[1:]:
            obj = self.component(obj, comp)
            if cargs is not None:
                obj = obj.get(self.subs(cargs, fr))
        if isinstance(obj, np.generic) and not isinstance(obj, np.void):
            obj = obj.item()
        return obj

    def component(self, obj, comp):
        if isinstance(obj, np.void):
            return obj[comp]
        if isinstance(obj, FArray) and obj.data.dtype.names:
            return FArray(obj.data[comp], obj.lb)
        return getattr(obj, comp)

    def assign(self, lhs, value, fr):
        parts = lhs[1]
        name, args = parts[0]
        scope, nm, ty = self.resolve(name, fr)
        if scope is None:
            raise FortranError(f"assignment to unknown {name}")
        if len(parts) == 1:
            if args is None:
                cur = scope[nm]
                if isinstance(cur, FArray):
                    cur.set([slice(None)] * cur.data.ndim, value if not isinstance(value, list) else np.array(value))
                else:
                    scope[nm] = self.convert(ty or ("integer" if is_int(cur) else "real"), value)
                return
            arr = scope[nm]
            idx = self.subs(args, fr)
            if isinstance(value, list):
                value = np.array(value)
            if arr.data.dtype.kind in "iu" and not isinstance(value, np.ndarray):
                value = int(value)
            arr.set(idx, value)
            return
        # component assignment: walk to the container of the last component
        obj = scope[nm]
        if args is not None:
            idx = self.subs(args, fr)
            if isinstance(obj, FArray) and obj.data.dtype.names and len(parts) == 2 and parts[1][1] is None:
                comp = parts[1][0]
                fld = obj.data[comp]
                k = obj._key(idx)
                fld[k] = int(value) if fld.dtype.kind in "iu" else value
                return
            obj = obj.get(idx)
        for comp, cargs in parts[1:-1]:
            obj = self.component(obj, comp)
            if cargs is not None:
                obj = obj.get(self.subs(cargs, fr))
        comp, cargs = parts[-1]
        if cargs is None:
            if isinstance(obj, DerivedObj):
                setattr(obj, comp, value)
            else:
                obj[comp] = value
        else:
            target = self.component(obj, comp)
            if isinstance(value, list):
                value = np.array(value)
            target.set(self.subs(cargs, fr), value)
