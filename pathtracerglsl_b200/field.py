"""Position-dependent medium coefficients: a GLSL expression of ``p`` compiled to a stack
program the device and the oracle interpret (heterogeneous media, the reference's
``{kind: 'glsl', source, params}`` coefficients of types.ts MediumDescription).

The accepted language is the expression subset the reference's media formulas use:
float literals, ``p`` and its components (``p.x`` ...), ``vec3(...)`` constructors, the
uniforms ``u_<param with '.' -> '_'>`` of the declared params (resolved to constants
at compile time), unary minus, ``+ - * /`` with GLSL precedence and scalar/vec3
broadcasting, component access on any vec3 term, and the built-ins exp, log, sin, cos,
sqrt, abs, floor, fract, pow, min, max, mod, step, clamp, mix, smoothstep, dot, length.
Every stack slot holds three floats; a scalar is kept broadcast, so component-wise
built-ins need no scalar forms.  The compiler tracks which terms are scalars to type
dot/length/vec3 and to reject what GLSL would reject.
"""
import re
import struct

from . import abi

OPS = {name: i for i, name in enumerate([
    "END", "CONST", "P", "SWZ", "ADD", "SUB", "MUL", "DIV", "NEG", "EXP", "LOG", "SIN", "COS", "SQRT",
    "ABS", "FLOOR", "FRACT", "POW", "MIN", "MAX", "MOD", "STEP", "CLAMP", "MIX", "SMOOTHSTEP", "DOT",
    "LENGTH", "VEC3"])}
MAX_STACK = 16
# built-in -> (opcode, arity)
FUNCS = {"exp": ("EXP", 1), "log": ("LOG", 1), "sin": ("SIN", 1), "cos": ("COS", 1), "sqrt": ("SQRT", 1),
         "abs": ("ABS", 1), "floor": ("FLOOR", 1), "fract": ("FRACT", 1), "pow": ("POW", 2), "min": ("MIN", 2),
         "max": ("MAX", 2), "mod": ("MOD", 2), "step": ("STEP", 2), "clamp": ("CLAMP", 3), "mix": ("MIX", 3),
         "smoothstep": ("SMOOTHSTEP", 3), "dot": ("DOT", 2), "length": ("LENGTH", 1)}
_TOKEN = re.compile(r"\s*(?:(\d+\.\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?|\d+(?:[eE][+-]?\d+)?)|([A-Za-z_]\w*)|(.))")


class FieldError(ValueError):
    pass


def _f32_bits(x):
    return struct.unpack("<I", struct.pack("<f", float(x)))[0]


class _Parser:
    def __init__(self, src, uniforms):
        self.toks = []
        pos = 0
        src = src.strip()
        while pos < len(src):
            m = _TOKEN.match(src, pos)
            if not m or m.end() == pos:
                raise FieldError(f"cannot read the expression at {src[pos:]!r}")
            num, ident, ch = m.groups()
            if num is not None:
                self.toks.append(("num", float(num)))
            elif ident is not None:
                self.toks.append(("id", ident))
            elif ch is not None and not ch.isspace():
                self.toks.append(("op", ch))
            pos = m.end()
        self.i = 0
        self.uniforms = uniforms
        self.code = []
        self.depth = 0
        self.max_depth = 0

    def peek(self):
        return self.toks[self.i] if self.i < len(self.toks) else ("end", None)

    def take(self, kind=None, val=None):
        t = self.peek()
        if (kind and t[0] != kind) or (val is not None and t[1] != val):
            raise FieldError(f"expected {val or kind}, found {t[1]!r}")
        self.i += 1
        return t

    def emit(self, op, *imm, push=0):
        self.code.append(OPS[op])
        self.code.extend(imm)
        self.depth += push
        self.max_depth = max(self.max_depth, self.depth)
        if self.max_depth > MAX_STACK:
            raise FieldError(f"expression nests deeper than {MAX_STACK} terms")

    def const(self, v):
        vals = list(v) if isinstance(v, (list, tuple)) else [v, v, v]
        self.emit("CONST", *[_f32_bits(x) for x in vals], push=1)

    # grammar: sum := prod (('+'|'-') prod)* ; prod := unary (('*'|'/') unary)* ;
    # unary := '-' unary | postfix ; postfix := atom ('.' swizzle)*
    def sum(self):
        s = self.prod()
        while self.peek() in (("op", "+"), ("op", "-")):
            op = self.take()[1]
            t = self.prod()
            self.emit("ADD" if op == "+" else "SUB", push=-1)
            s = s and t
        return s

    def prod(self):
        s = self.unary()
        while self.peek() in (("op", "*"), ("op", "/")):
            op = self.take()[1]
            t = self.unary()
            self.emit("MUL" if op == "*" else "DIV", push=-1)
            s = s and t
        return s

    def unary(self):
        if self.peek() == ("op", "-"):
            self.take()
            s = self.unary()
            self.emit("NEG")
            return s
        if self.peek() == ("op", "+"):
            self.take()
            return self.unary()
        return self.postfix()

    def postfix(self):
        s = self.atom()
        while self.peek() == ("op", "."):
            self.take()
            comp = self.take("id")[1]
            if s or comp not in ("x", "y", "z", "r", "g", "b"):
                raise FieldError(f"component access .{comp} needs a vec3 and one of x, y, z")
            self.emit("SWZ", "xyzrgb".index(comp) % 3)
            s = True
        return s

    def atom(self):
        kind, val = self.peek()
        if kind == "num":
            self.take()
            self.const(val)
            return True
        if kind == "op" and val == "(":
            self.take()
            s = self.sum()
            self.take("op", ")")
            return s
        if kind == "id":
            self.take()
            if val == "p":
                self.emit("P", push=1)
                return False
            if val in self.uniforms:
                u = self.uniforms[val]
                self.const(u)
                return not isinstance(u, (list, tuple))
            if val in ("vec3",) or val in FUNCS:
                self.take("op", "(")
                args = [self.sum()]
                while self.peek() == ("op", ","):
                    self.take()
                    args.append(self.sum())
                self.take("op", ")")
                return self.call(val, args)
            raise FieldError(f"unknown name {val!r} (p, u_<param>, vec3 and {', '.join(sorted(FUNCS))} are known)")
        raise FieldError(f"unexpected {val!r}")

    def call(self, name, scal):
        n = len(scal)
        if name == "vec3":
            if n == 1:
                return False          # vec3(s): the broadcast scalar is already a vec3
            if n != 3 or not all(scal):
                raise FieldError("vec3(...) takes one scalar or three scalars")
            self.emit("VEC3", push=-2)
            return False
        op, arity = FUNCS[name]
        if n != arity:
            raise FieldError(f"{name} takes {arity} arguments, not {n}")
        if name == "dot":
            if scal[0] != scal[1]:
                raise FieldError("dot of a scalar and a vec3")
            if scal[0]:
                self.emit("MUL", push=-1)
            else:
                self.emit("DOT", push=-1)
            return True
        if name == "length":
            if scal[0]:
                self.emit("ABS")
            else:
                self.emit("LENGTH")
            return True
        self.emit(op, push=1 - arity)
        return all(scal)


def compile_field(expr, params):
    """Bytecode words (uint32, END-terminated) of a ``{kind: 'glsl', source, params}``
    coefficient, its uniforms resolved from ``params`` (param name -> value) or their
    declared defaults."""
    if not (isinstance(expr, dict) and expr.get("kind") == "glsl" and isinstance(expr.get("source"), str)):
        raise FieldError("a medium expression is {kind: 'glsl', source: str, params: [...]}")
    uniforms = {}
    for decl in expr.get("params", []):
        name = decl["param"]
        uniforms["u_" + name.replace(".", "_")] = params.get(name, decl.get("default", 0.0))
    ps = _Parser(expr["source"], uniforms)
    ps.sum()
    if ps.peek()[0] != "end":
        raise FieldError(f"unexpected {ps.peek()[1]!r} after the expression")
    ps.emit("END")
    return ps.code


def is_field(v):
    return isinstance(v, dict) and v.get("kind") == "glsl"


assert abi.FIELD_MAX_STACK == MAX_STACK
