"""Mechanical Fortran-90 -> C translation of the reference solver (oracle pin).

TEST INFRASTRUCTURE ONLY.  No Fortran compiler exists on this machine, so
this script compiles the reference's own active source files (read from the
reference checkout given on the command line; nothing is copied into the
repository) into C, written to oracle/_ref/ref_translated.c.  Together with
oracle/ref_runtime.c it builds oracle/_ref/libref.so, which the tests run on
the same inputs as the C++ oracle and compare bit for bit.

It handles exactly the Fortran subset the reference uses: modules with
module variables, one derived type, allocatable arrays, subroutines with
by-reference arguments, DO / IF blocks, whole-array and section assignments,
list-directed READ (with an implied-DO), and the intrinsics dsqrt, dexp,
dlog, derf, dabs, datan, dcos, dsin, dlog10.  Semantics follow gfortran on
x86-64: left-to-right evaluation, no contraction (build with
-ffp-contract=off), REAL*4 literals such as 0.5 or 10e-6 are single-precision
values widened to double, x**2 is x*x and a real exponent calls pow().

Memory model: every array is 1-based, column-major, and allocated with a
zero-filled guard of GUARD elements on both sides, so the reference's
out-of-range accesses (point_with_alias(N) = 0 used as an index; split lists
written past their 22-entry capacity) behave as unchecked Fortran indexing
into zeroed memory does, without touching other arrays' storage.
Compile-time PARAMETERs become variables so a run can set max_points, Mach
and the angle of attack; their defining expressions are evaluated at start.

usage: python f2c_ref.py REFERENCE_DIR OUT_C [VARIANT ...]
"""
from __future__ import annotations

import os
import re
import sys

GUARD = 256

ACTIVE_FILES = [
    "parameter.f90", "data_structure.f90", "point_preprocessor.f90", "initial_conditions.f90",
    "generate_connectivity.f90", "implicit_aliasing.f90", "compute_conserved_vector.f90",
    "q_variables.f90", "q_derivatives.f90", "timestep_delt.f90", "limiters.f90",
    "qvariables_to_primitive_variables.f90", "split_fluxes.f90", "octant_fluxes.f90",
    "interior_flux_dGxpos.f90", "interior_flux_dGxneg.f90", "interior_flux_dGypos.f90",
    "interior_flux_dGyneg.f90", "interior_flux_dGzpos.f90", "interior_flux_dGzneg.f90",
    "wall_flux_dGxpos.f90", "wall_flux_dGxneg.f90", "wall_flux_dGypos.f90",
    "wall_flux_dGyneg.f90", "wall_flux_dGzneg.f90",
    "outer_flux_dGxpos.f90", "outer_flux_dGxneg.f90", "outer_flux_dGypos.f90",
    "outer_flux_dGyneg.f90", "outer_flux_dGzpos.f90", "flux_residual.f90",
    "get_primitive_vector.f90", "conserved_to_primitive_vector.f90", "conserved_vector_Ubar.f90",
    "implicit_D_inv_interior.f90", "implicit_D_inv_wall.f90", "implicit_D_inv_outer.f90",
    "implicit_LdelU_forward_sweep_interior.f90", "implicit_LdelU_forward_sweep_wall.f90",
    "implicit_LdelU_forward_sweep_outer.f90", "implicit_UdelU_backward_sweep_interior.f90",
    "implicit_UdelU_backward_sweep_wall.f90", "implicit_UdelU_backward_sweep_outer.f90",
    "implicit_forward_and_reverse_sweeps.f90", "state_update_implicit.f90", "fpi_solver.f90",
]

INTRINSICS = {"dsqrt": "sqrt", "sqrt": "sqrt", "dexp": "exp", "exp": "exp", "dlog": "log",
              "log": "log", "derf": "erf", "erf": "erf", "dabs": "fabs", "abs": "fabs",
              "datan": "atan", "dcos": "cos", "dsin": "sin", "dlog10": "log10"}

TYPE_RANK = {"int": 0, "r4": 1, "r8": 2, "log": -1}
CTYPE = {"int": "int", "r4": "float", "r8": "double", "log": "int"}


class F2CError(Exception):
    pass


# ------------------------------------------------------------------ lexing

TOKEN_RE = re.compile(r"""
   (?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eEdD][+-]?\d+)?)
 | (?P<dotop>\.(?:le|lt|ge|gt|eq|ne|and|or|not|true|false)\.)
 | (?P<name>[a-zA-Z_][a-zA-Z_0-9]*)
 | (?P<str>'[^']*'|"[^"]*")
 | (?P<op>\*\*|==|/=|<=|>=|::|[-+*/(),=<>%:])
 | (?P<ws>\s+)
""", re.X | re.I)


def tokenize(s):
    out, i = [], 0
    while i < len(s):
        m = TOKEN_RE.match(s, i)
        if not m:
            raise F2CError(f"cannot tokenize: {s[i:i + 30]!r}")
        kind = m.lastgroup
        if kind in ("dotop", "name", "num"):
            out.append((kind, m.group(kind).lower()))
        elif kind != "ws":
            out.append((kind, m.group(kind)))
        i = m.end()
    return out


def logical_lines(text):
    """Free-form source -> statements (comments stripped, continuations joined)."""
    stmts, buf = [], ""
    for raw in text.splitlines():
        line, q = "", None
        for ch in raw:
            if q:
                line += ch
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
                line += ch
            elif ch == "!":
                break
            else:
                line += ch
        line = line.strip()
        if buf and line.startswith("&"):
            line = line[1:].strip()
        if line.endswith("&"):
            buf += line[:-1] + " "
            continue
        line = buf + line
        buf = ""
        if line:
            stmts.append(line)
    return stmts


# ------------------------------------------------------------------ expressions

class P:
    """Recursive-descent parser over one token list."""

    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k] if self.i + k < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise F2CError(f"expected {val!r}, got {tok[1]!r} in {self.rest()}")
        self.i += 1
        return tok

    def rest(self):
        return " ".join(v for _, v in self.t[self.i:])

    def at_end(self):
        return self.i >= len(self.t)

    # precedence climbing, Fortran rules
    def expr(self):
        return self.or_()

    def or_(self):
        a = self.and_()
        while self.peek()[1] == ".or.":
            self.take()
            a = ("bin", "||", a, self.and_())
        return a

    def and_(self):
        a = self.not_()
        while self.peek()[1] == ".and.":
            self.take()
            a = ("bin", "&&", a, self.not_())
        return a

    def not_(self):
        if self.peek()[1] == ".not.":
            self.take()
            return ("not", self.not_())
        return self.rel()

    REL = {".le.": "<=", ".lt.": "<", ".ge.": ">=", ".gt.": ">", ".eq.": "==", ".ne.": "!=",
           "<=": "<=", "<": "<", ">=": ">=", ">": ">", "==": "==", "/=": "!="}

    def rel(self):
        a = self.add()
        op = self.peek()[1]
        if op in self.REL:
            self.take()
            return ("rel", self.REL[op], a, self.add())
        return a

    def add(self):
        sign = None
        if self.peek()[1] in ("+", "-"):
            sign = self.take()[1]
        a = self.mul()
        if sign == "-":
            a = ("neg", a)
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = ("bin", op, a, self.mul())
        return a

    def mul(self):
        a = self.power()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            a = ("bin", op, a, self.power())
        return a

    def power(self):
        a = self.primary()
        if self.peek()[1] == "**":
            self.take()
            return ("pow", a, self.power())      # right associative
        return a

    def primary(self):
        kind, val = self.peek()
        if val == "(":
            self.take()
            e = self.expr()
            self.take(")")
            return ("paren", e)
        if kind == "num":
            self.take()
            return ("num", val)
        if kind == "name":
            return self.designator()
        raise F2CError(f"unexpected token {val!r} in {self.rest()}")

    def designator(self):
        _, name = self.take()
        node = ("name", name.lower(), None)
        if self.peek()[1] == "%":
            self.take()
            _, comp = self.take()
            node = ("comp", name.lower(), comp.lower(), None)
        if self.peek()[1] == "(":
            self.take()
            subs = []
            if self.peek()[1] != ")":
                while True:
                    subs.append(self.subscript())
                    if self.peek()[1] == ",":
                        self.take()
                        continue
                    break
            self.take(")")
            node = node[:-1] + (subs,)
        return node

    def subscript(self):
        if self.peek()[1] == ":":
            self.take()
            return ("colon",)
        return self.expr()


# ------------------------------------------------------------------ symbols

class Sym:
    def __init__(self, name, base, rank=0, dims=None, kind="local", cname=None, alloc=False):
        self.name, self.base, self.rank, self.dims = name, base, rank, dims or []
        self.kind, self.cname, self.alloc = kind, cname, alloc
        self.init = None


def parse_type(tokens):
    """Leading type spec -> (base, rest tokens)."""
    v = [t[1].lower() for t in tokens]
    if v[0] == "integer":
        return "int", tokens[1:]
    if v[0] == "double" and v[1] == "precision":
        return "r8", tokens[2:]
    if v[0] == "real":
        if len(v) > 2 and v[1] == "*" and v[2] == "8":
            return "r8", tokens[3:]
        if len(v) > 2 and v[1] == "*" and v[2] == "4":
            return "r4", tokens[3:]
        return "r4", tokens[1:]
    if v[0] == "logical":
        return "log", tokens[1:]
    raise F2CError("unknown type " + " ".join(v))


def split_top(tokens, sep=","):
    out, cur, depth = [], [], 0
    for t in tokens:
        if t[1] == "(":
            depth += 1
        elif t[1] == ")":
            depth -= 1
        if t[1] == sep and depth == 0:
            out.append(cur)
            cur = []
        else:
            cur.append(t)
    if cur:
        out.append(cur)
    return out


def parse_decl(tokens):
    """-> (base, attrs, [(name, dims or None, init tokens or None)])"""
    base, rest = parse_type(tokens)
    attrs, dim_attr = [], None
    vals = [t[1].lower() for t in rest]
    if "::" in vals:
        k = vals.index("::")
        attr_toks, ent_toks = rest[:k], rest[k + 1:]
        for a in split_top(attr_toks):
            if not a:
                continue
            an = a[0][1].lower()
            if an == "dimension":
                dim_attr = [d for d in split_top(a[2:-1])]
            attrs.append(an)
    else:
        ent_toks = rest
    ents = []
    for e in split_top(ent_toks):
        name = e[0][1].lower()
        dims, init = None, None
        j = 1
        if j < len(e) and e[j][1] == "(":
            depth, k = 0, j
            while True:
                if e[k][1] == "(":
                    depth += 1
                elif e[k][1] == ")":
                    depth -= 1
                    if depth == 0:
                        break
                k += 1
            dims = split_top(e[j + 1:k])
            j = k + 1
        if j < len(e) and e[j][1] == "=":
            init = e[j + 1:]
        ents.append((name, dims if dims is not None else dim_attr, init))
    return base, attrs, ents


# ------------------------------------------------------------------ program model

class Sub:
    def __init__(self, name, args, module):
        self.name, self.args, self.module = name, args, module
        self.syms = {}
        self.body = []


class Translator:
    def __init__(self):
        self.globals = {}            # module variables and parameters
        self.type_comps = {}         # component name -> Sym (of the single derived type)
        self.type_var = None         # name of the derived-type variable ("point")
        self.params = []             # parameter Syms in declaration order
        self.subs = {}
        self.out = []

    # ---- pass 1: declarations and statement lists
    def load(self, path):
        text = open(path).read()
        stmts = logical_lines(text)
        module, sub, in_type = None, None, False
        for s in stmts:
            toks = tokenize(s)
            low = [t[1].lower() for t in toks]
            head = low[0]
            if head == "module" and len(low) == 2:
                module = low[1]
                continue
            if head == "end" and len(low) >= 2 and low[1] == "module":
                module = None
                continue
            if head in ("use", "implicit", "contains"):
                continue
            if head == "type" and "::" in low and "(" not in low[:2]:
                in_type = True
                continue
            if head == "end" and len(low) >= 2 and low[1] == "type":
                in_type = False
                continue
            if head == "type" and low[1] == "(":
                # type(points) :: point
                self.type_var = low[-1]
                continue
            if head == "subroutine":
                name = low[1]
                args = [a for a in low[3:-1] if a != ","] if "(" in low else []
                sub = Sub(name, args, module)
                self.subs[name] = sub
                continue
            if head == "end" and (len(low) == 1 or low[1] == "subroutine"):
                sub = None
                continue
            if head in ("integer", "real", "double", "logical"):
                base, attrs, ents = parse_decl(toks)
                for name, dims, init in ents:
                    if in_type:
                        self.type_comps[name] = Sym(name, base, len(dims) if dims else 0, None,
                                                    "comp", "pc_" + name, alloc=True)
                    elif sub is not None:
                        kind = "dummy" if name in sub.args else "local"
                        sy = Sym(name, base, len(dims) if dims else 0,
                                 [d for d in dims] if dims else [], kind, "v_" + name)
                        sub.syms[name] = sy
                    else:
                        sy = Sym(name, base, len(dims) if dims else 0, None, "module",
                                 "m_" + name, alloc="allocatable" in attrs)
                        if "parameter" in attrs:
                            sy.kind = "param"
                            sy.init = init
                            self.params.append(sy)
                        self.globals[name] = sy
                continue
            if sub is None:
                raise F2CError(f"{path}: statement outside a subroutine: {s}")
            sub.body.append(toks)

    # ---- helpers
    def lookup(self, sub, name):
        if sub is not None and name in sub.syms:
            return sub.syms[name]
        if name in self.globals:
            return self.globals[name]
        raise F2CError(f"unknown name {name!r} in {sub.name if sub else '?'}")

    def dims_c(self, sub, sym):
        """C expressions for each dimension's extent."""
        if sym.kind == "comp" or sym.alloc:
            return [f"{sym.cname}_d[{k}]" for k in range(sym.rank)]
        return [self.expr_c(sub, P(d).expr(), [])[0] for d in sym.dims]

    def elem_ref(self, sub, sym, subs, loopvars, lv_pos):
        """C lvalue for one element; ':' subscripts take loop variables."""
        dims = self.dims_c(sub, sym)
        idx = []
        for k in range(sym.rank):
            s = subs[k] if subs is not None else ("colon",)
            if s[0] == "colon":
                idx.append(f"({loopvars[lv_pos[0]]})")
                lv_pos[0] += 1
            else:
                c, t = self.expr_c(sub, s, [])
                idx.append(f"({c})")
        off = f"({idx[-1]} - 1)"
        for k in range(sym.rank - 2, -1, -1):
            off = f"({idx[k]} - 1 + (long)({dims[k]}) * {off})"
        base = f"(*{sym.cname})" if False else sym.cname
        return f"{base}[{off}]"

    def section_rank(self, node, sub):
        kind = node[0]
        if kind in ("name", "comp"):
            sym = self.sym_of(node, sub)
            subs = node[-1]
            if sym is None:
                return 0
            if sym.rank == 0:
                return 0
            if subs is None:
                return sym.rank
            return sum(1 for s in subs if s[0] == "colon")
        if kind in ("bin", "rel"):
            return max(self.section_rank(node[2], sub), self.section_rank(node[3], sub))
        if kind in ("neg", "not", "paren"):
            return self.section_rank(node[1], sub)
        if kind == "pow":
            return max(self.section_rank(node[1], sub), self.section_rank(node[2], sub))
        return 0

    def sym_of(self, node, sub):
        if node[0] == "comp":
            return self.type_comps[node[2]]
        name = node[1]
        if name in INTRINSICS and (sub is None or name not in sub.syms) and name not in self.globals:
            return None
        return self.lookup(sub, name)

    def section_extents(self, node, sub):
        sym = self.sym_of(node, sub)
        dims = self.dims_c(sub, sym)
        subs = node[-1]
        if subs is None:
            return dims
        return [dims[k] for k, s in enumerate(subs) if s[0] == "colon"]

    def first_array(self, node, sub):
        kind = node[0]
        if kind in ("name", "comp"):
            sym = self.sym_of(node, sub)
            if sym is not None and self.section_rank(node, sub) > 0:
                return node
            if sym is None and node[-1]:
                for a in node[-1]:
                    r = self.first_array(a, sub)
                    if r:
                        return r
            return None
        for child in node[1:]:
            if isinstance(child, tuple):
                r = self.first_array(child, sub)
                if r:
                    return r
        return None

    # ---- expressions -> (code, type)
    def expr_c(self, sub, node, loopvars):
        kind = node[0]
        if kind == "num":
            v = node[1].lower()
            if re.fullmatch(r"\d+", v):
                return v, "int"
            if "d" in v:
                return "(" + v.replace("d", "e") + ")", "r8"
            lit = v if ("e" in v or "." in v) else v + ".0"
            if lit.endswith("."):
                lit += "0"
            return f"((double){lit}f)", "r4w"          # REAL*4 literal, widened on use
        if kind == "paren":
            c, t = self.expr_c(sub, node[1], loopvars)
            return f"({c})", t
        if kind == "neg":
            c, t = self.expr_c(sub, node[1], loopvars)
            return f"(-{c})", t
        if kind == "not":
            c, t = self.expr_c(sub, node[1], loopvars)
            return f"(!{c})", "log"
        if kind in ("bin", "rel"):
            a, ta = self.expr_c(sub, node[2], loopvars)
            b, tb = self.expr_c(sub, node[3], loopvars)
            op = node[1]
            if op in ("&&", "||"):
                return f"({a} {op} {b})", "log"
            t = self.promote(ta, tb)
            a, b = self.conv(a, ta, t), self.conv(b, tb, t)
            if kind == "rel":
                return f"({a} {op} {b})", "log"
            return f"({a} {op} {b})", t
        if kind == "pow":
            a, ta = self.expr_c(sub, node[1], loopvars)
            if node[2][0] == "num" and re.fullmatch(r"\d+", node[2][1]):
                n = int(node[2][1])
                if n == 2:
                    return f"(({a}) * ({a}))", ta
                if n == 3:
                    return f"((({a}) * ({a})) * ({a}))", ta
            b, tb = self.expr_c(sub, node[2], loopvars)
            return f"pow({self.conv(a, ta, 'r8')}, {self.conv(b, tb, 'r8')})", "r8"
        if kind in ("name", "comp"):
            sym = self.sym_of(node, sub)
            if sym is None:
                fn = INTRINSICS[node[1]]
                args = [self.expr_c(sub, a, loopvars) for a in node[2]]
                cargs = ", ".join(self.conv(c, t, "r8") for c, t in args)
                return f"{fn}({cargs})", "r8"
            if sym.rank == 0:
                if sym.kind == "dummy":
                    return f"(*{sym.cname})", sym.base
                return sym.cname, sym.base
            return self.elem_ref(sub, sym, node[-1], loopvars, [0]), sym.base
        raise F2CError(f"bad expression node {node}")

    @staticmethod
    def promote(ta, tb):
        def r(t):
            return {"int": 0, "r4": 1, "r4w": 1, "r8": 2, "log": -1}[t]
        if "r8" in (ta, tb):
            return "r8"
        if ta in ("r4", "r4w") and tb in ("r4", "r4w"):
            return "r4"
        if "r4" in (ta, tb) or "r4w" in (ta, tb):
            return "r4"
        return "int" if r(ta) >= 0 and r(tb) >= 0 else "log"

    @staticmethod
    def conv(code, t, to):
        if to == "r8":
            if t == "r8":
                return code
            if t == "r4w":          # single-precision literal widened: value of the float
                return code
            if t == "r4":
                return f"(double)({code})"
            return f"(double)({code})"
        if to == "r4":
            if t == "r4":
                return code
            return f"(float)({code})"
        if to == "int":
            if t == "int":
                return code
            return f"(int)({code})"
        return code

    # ---- statements
    def stmt_c(self, sub, toks, ind):
        low = [t[1].lower() for t in toks]
        head = low[0]
        pad = "    " * ind
        if head == "do" and len(low) > 1 and low[2] == "=":
            var = low[1]
            parts = split_top(toks[3:])
            a = self.expr_c(sub, P(parts[0]).expr(), [])[0]
            b = self.expr_c(sub, P(parts[1]).expr(), [])[0]
            step = self.expr_c(sub, P(parts[2]).expr(), [])[0] if len(parts) > 2 else "1"
            v = self.expr_c(sub, ("name", var, None), [])[0]
            cmp = "<=" if not step.startswith("(-") and not step.startswith("-") else ">="
            return [f"{pad}for ({v} = {a}; {v} {cmp} {b}; {v} += {step}) {{"], +1
        if head in ("enddo",) or (head == "end" and len(low) > 1 and low[1] == "do"):
            return [pad[:-4] + "}"], -1
        if head == "if":
            # find the matching ')'
            depth, k = 0, 1
            while True:
                if toks[k][1] == "(":
                    depth += 1
                elif toks[k][1] == ")":
                    depth -= 1
                    if depth == 0:
                        break
                k += 1
            cond = self.expr_c(sub, P(toks[2:k]).expr(), [])[0]
            tail = low[k + 1:]
            if tail == ["then"]:
                return [f"{pad}if ({cond}) {{"], +1
            inner, _ = self.stmt_c(sub, toks[k + 1:], ind + 1)
            return [f"{pad}if ({cond}) {{"] + inner + [f"{pad}}}"], 0
        if head == "else" and len(low) > 1 and low[1] == "if":
            inner = toks[1:]
            lines, _ = self.stmt_c(sub, inner, ind - 1)
            return [pad[:-4] + "} else " + lines[0].strip()], 0
        if head == "else":
            return [pad[:-4] + "} else {"], 0
        if head in ("endif",) or (head == "end" and len(low) > 1 and low[1] == "if"):
            return [pad[:-4] + "}"], -1
        if head == "call":
            return [pad + self.call_c(sub, toks)], 0
        if head in ("print", "write", "close"):
            return [pad + "/* " + " ".join(low[:3]) + " ... (output skipped) */"], 0
        if head == "open":
            unit = file = None
            for kv in split_top(toks[2:-1]):
                key = kv[0][1].lower()
                if key == "unit":
                    unit = kv[2][1]
                elif key == "file":
                    file = kv[2][1]
            return [f"{pad}ref_open({unit}, {file.replace(chr(39), chr(34))});"], 0
        if head == "read":
            return self.read_c(sub, toks, pad), 0
        if head == "allocate":
            return self.allocate_c(sub, toks, pad), 0
        if "=" in low:
            return self.assign_c(sub, toks, pad), 0
        raise F2CError(f"unsupported statement in {sub.name}: {' '.join(low)}")

    def assign_c(self, sub, toks, pad):
        k = [t[1] for t in toks].index("=")
        lhs = P(toks[:k]).designator()
        rhs = P(toks[k + 1:]).expr()
        sym = self.sym_of(lhs, sub)
        rank = self.section_rank(lhs, sub)
        if rank == 0:
            lc, lt = self.expr_c(sub, lhs, [])
            rc, rt = self.expr_c(sub, rhs, [])
            return [f"{pad}{lc} = {self.conv(rc, rt, sym.base)};"]
        ext = self.section_extents(lhs, sub)
        lvs = [f"_e{j}" for j in range(rank)]
        lines = [f"{pad}{{"]
        for j, (lv, e) in enumerate(zip(lvs, ext)):
            lines.append(f"{pad}  for (long {lv} = 1; {lv} <= ({e}); ++{lv})")
        lc, _ = self.expr_c(sub, lhs, lvs)
        rc, rt = self.expr_c_elemental(sub, rhs, lvs)
        lines.append(f"{pad}    {lc} = {self.conv(rc, rt, sym.base)};")
        lines.append(f"{pad}}}")
        return lines

    def expr_c_elemental(self, sub, node, lvs):
        """Like expr_c, but array operands (sections or whole arrays) take the loop variables."""
        kind = node[0]
        if kind in ("name", "comp"):
            sym = self.sym_of(node, sub)
            if sym is not None and self.section_rank(node, sub) > 0:
                return self.elem_ref(sub, sym, node[-1], lvs, [0]), sym.base
            if sym is None:
                fn = INTRINSICS[node[1]]
                args = [self.expr_c_elemental(sub, a, lvs) for a in node[2]]
                return f"{fn}({', '.join(self.conv(c, t, 'r8') for c, t in args)})", "r8"
            return self.expr_c(sub, node, [])
        if kind == "num":
            return self.expr_c(sub, node, [])
        if kind == "paren":
            c, t = self.expr_c_elemental(sub, node[1], lvs)
            return f"({c})", t
        if kind == "neg":
            c, t = self.expr_c_elemental(sub, node[1], lvs)
            return f"(-{c})", t
        if kind in ("bin", "rel"):
            a, ta = self.expr_c_elemental(sub, node[2], lvs)
            b, tb = self.expr_c_elemental(sub, node[3], lvs)
            t = self.promote(ta, tb)
            op = node[1]
            if kind == "rel":
                return f"({self.conv(a, ta, t)} {op} {self.conv(b, tb, t)})", "log"
            return f"({self.conv(a, ta, t)} {op} {self.conv(b, tb, t)})", t
        if kind == "pow":
            return self.expr_c(sub, node, [])
        raise F2CError(f"bad elemental node {node}")

    def call_c(self, sub, toks):
        name = toks[1][1].lower()
        callee = self.subs.get(name)
        if callee is None:
            raise F2CError(f"call of unknown subroutine {name}")
        args = split_top(toks[3:-1]) if len(toks) > 3 else []
        cargs = []
        for a, dummy in zip(args, callee.args):
            dsym = callee.syms[dummy]
            node = P(a).expr()
            if node[0] not in ("name", "comp"):
                raise F2CError(f"non-variable actual argument in call {name}")
            asym = self.sym_of(node, sub)
            if dsym.rank > 0:
                if node[-1] is None:
                    cargs.append(asym.cname if asym.kind != "dummy" else asym.cname)
                else:
                    ones = [("num", "1") if s[0] == "colon" else s for s in node[-1]]
                    cargs.append("&" + self.elem_ref(sub, asym, ones, [], [0]))
            else:
                if asym.rank == 0:
                    cargs.append(asym.cname if asym.kind == "dummy" else "&" + asym.cname)
                else:
                    cargs.append("&" + self.elem_ref(sub, asym, node[-1], [], [0]))
        return f"f_{name}({', '.join(cargs)});"

    def read_c(self, sub, toks, pad):
        # read(unit,*) item, item, (item, var=a,b), ...
        close = [t[1] for t in toks].index(")")
        unit = toks[2][1]
        items = split_top(toks[close + 1:])
        lines = [f"{pad}ref_read_begin({unit});"]
        for it in items:
            if it[0][1] == "(":
                inner = split_top(it[1:-1])
                var = inner[1][0][1].lower()
                lo = self.expr_c(sub, P(inner[1][2:]).expr(), [])[0]
                hi = self.expr_c(sub, P(inner[2]).expr(), [])[0]
                vc = self.expr_c(sub, ("name", var, None), [])[0]
                node = P(inner[0]).designator()
                lc, lt = self.expr_c(sub, node, [])
                fn = "ref_read_int" if lt == "int" else "ref_read_dbl"
                lines.append(f"{pad}for ({vc} = {lo}; {vc} <= {hi}; ++{vc}) {fn}(&{lc});")
            else:
                node = P(it).designator()
                lc, lt = self.expr_c(sub, node, [])
                fn = "ref_read_int" if lt == "int" else "ref_read_dbl"
                lines.append(f"{pad}{fn}(&{lc});")
        lines.append(f"{pad}ref_read_end({unit});")
        return lines

    def allocate_c(self, sub, toks, pad):
        lines = []
        for item in split_top(toks[2:-1]):
            node = P(item).designator()
            sym = self.sym_of(node, sub)
            dims = [self.expr_c(sub, d, [])[0] for d in node[-1]]
            total = " * ".join(f"(long)({d})" for d in dims)
            alloc = "ref_alloc_int" if sym.base == "int" else "ref_alloc_dbl"
            for k, dd in enumerate(dims):
                lines.append(f"{pad}{sym.cname}_d[{k}] = {dd};")
            lines.append(f"{pad}{sym.cname} = {alloc}({total});")
        return lines

    # ---- emit
    def emit(self):
        o = self.out
        o.append("/* Generated by oracle/f2c_ref.py from the reference's Fortran sources. */")
        o.append("#include <math.h>")
        o.append('#include "../ref_runtime.h"')
        o.append("")
        for sy in self.params:
            o.append(f"{CTYPE[sy.base]} {sy.cname};")
        for name, sy in self.globals.items():
            if sy.kind == "param":
                continue
            if sy.alloc:
                o.append(f"{CTYPE[sy.base]} *{sy.cname}; long {sy.cname}_d[{max(sy.rank, 1)}];")
            else:
                o.append(f"{CTYPE[sy.base]} {sy.cname};")
        for name, sy in self.type_comps.items():
            o.append(f"{CTYPE[sy.base]} *{sy.cname}; long {sy.cname}_d[{max(sy.rank, 1)}];")
        o.append("")
        # parameters: defining expressions, evaluated in order; overrides applied by the runtime
        o.append("void ref_init_parameters(void) {")
        for sy in self.params:
            c, t = self.expr_c(None, P(sy.init).expr(), [])
            o.append(f"    if (!ref_param_overridden(\"{sy.name}\")) {sy.cname} = {self.conv(c, t, sy.base)};")
            o.append(f"    else {sy.cname} = ({CTYPE[sy.base]})ref_param_value(\"{sy.name}\");")
        o.append("}")
        o.append("")
        for s in self.subs.values():
            o.append(self.proto(s) + ";")
        o.append("")
        for s in self.subs.values():
            o.append(self.proto(s) + " {")
            for name, sy in s.syms.items():
                if sy.kind == "dummy":
                    continue
                if sy.rank == 0:
                    o.append(f"    {CTYPE[sy.base]} {sy.cname} = 0;")
                else:
                    n = " * ".join(f"({self.expr_c(s, P(d).expr(), [])[0]})" for d in sy.dims)
                    o.append(f"    {CTYPE[sy.base]} {sy.cname}_store[{n}] = {{0}};")
                    o.append(f"    {CTYPE[sy.base]} *{sy.cname} = {sy.cname}_store;")
            ind = 1
            for toks in s.body:
                lines, delta = self.stmt_c(s, toks, ind)
                o.extend(lines)
                ind += delta
            if ind != 1:
                raise F2CError(f"unbalanced blocks in {s.name}")
            o.append("}")
            o.append("")
        # exported entry points
        o.append("void ref_call(const char *name) {")
        for s in self.subs.values():
            if not s.args:
                o.append(f"    if (!ref_strcmp(name, \"{s.name}\")) {{ f_{s.name}(); return; }}")
        o.append("    ref_unknown_call(name);")
        o.append("}")
        o.append("void ref_fpi_solver(int t) { int tt = t; f_fpi_solver(&tt); }")
        o.append("void *ref_array(const char *name, long *dims) {")
        for name, sy in list(self.type_comps.items()) + [(n, s) for n, s in self.globals.items() if s.alloc]:
            o.append(f"    if (!ref_strcmp(name, \"{name}\")) {{ for (int k = 0; k < {max(sy.rank, 1)}; ++k) dims[k] = {sy.cname}_d[k]; return {sy.cname}; }}")
        o.append("    return 0;")
        o.append("}")
        o.append("double ref_scalar(const char *name) {")
        for name, sy in self.globals.items():
            if not sy.alloc:
                o.append(f"    if (!ref_strcmp(name, \"{name}\")) return (double){sy.cname};")
        o.append("    return 0.0 / 0.0;")
        o.append("}")
        o.append("void ref_set_scalar(const char *name, double v) {")
        for name, sy in self.globals.items():
            if not sy.alloc:
                o.append(f"    if (!ref_strcmp(name, \"{name}\")) {{ {sy.cname} = ({CTYPE[sy.base]})v; return; }}")
        o.append("}")
        return "\n".join(o) + "\n"

    def proto(self, s):
        parts = []
        for a in s.args:
            sy = s.syms[a]
            parts.append(f"{CTYPE[sy.base]} *{sy.cname}")
        return f"static void f_{s.name}({', '.join(parts) if parts else 'void'})"


# Alternative source files of the same modules (the reference compiles one of
# each pair): name -> (active file, replacement)
VARIANTS = {
    "explicit": ("state_update_implicit.f90", "state_update.f90"),
    "backup": ("implicit_forward_and_reverse_sweeps.f90", "implicit_forward_and_reverse_sweeps_backup.f90"),
}


def main():
    ref_dir, out_c = sys.argv[1], sys.argv[2]
    files = list(ACTIVE_FILES)
    for v in sys.argv[3:]:                 # optional variant names
        old, new = VARIANTS[v]
        files[files.index(old)] = new
    tr = Translator()
    for f in files:
        tr.load(os.path.join(ref_dir, f))
    src = tr.emit()
    os.makedirs(os.path.dirname(os.path.abspath(out_c)), exist_ok=True)
    with open(out_c, "w") as fh:
        fh.write(src)
    print(f"translated {len(files)} files, {len(tr.subs)} subroutines -> {out_c}")


if __name__ == "__main__":
    main()
