"""Material files of the reference's material library (mat_lib/*.lua) without
a Lua interpreter.

The files are Lua scripts run by the reference's material loader
(src/materials/lua_material.cpp:387-497): a fresh Lua state with the
standard libraries, the loader's functions registered as globals acting on
one Material (reset first, material.cpp:608-640), and the script run under
lua_pcall, so the first error stops the script silently and the material
keeps what it had by then. The library's files use a small part of Lua:
assignments to names, arithmetic on numbers, string literals, the math
library and calls of the loader's functions. This module reads exactly that
part (anything else is reported as outside it) and applies the calls with the
loader's meaning (lua_material.cpp:100-380):

  epsilon_infty / epsilon_infinity(e)   eps_inf = e
  index_infty / index_infinity(n)       eps_inf = n * n
  refractive_index(n)                   eps_inf = n * n (Material::set_const_n)
  add_debye(ds, t0), add_drude(wd, g), add_lorentz(A, O, G),
  add_crit_point(A, O, P, G)            one term each, in call order
  add_cauchy(...), add_sellmeier(B, C), add_data_index(...),
  add_data_epsilon(...)                 models the FDTD cannot run
  add_effective_component, effective_host, effective_type
                                        effective-medium materials (likewise)
  name(s), description(s), validity_range(a, b)
  load_script(path)                     loads another file into the material

Values are numbers, strings and lists ({a, b, ...}, the tabulated files'
vectors).

A material is usable by the FDTD when Material::fdtd_compatible holds
(material.cpp:147-158): no Cauchy, Sellmeier or tabulated (spline) data and
not an effective medium. FDTD_Material::set_base_mat (mats.cpp:445-464)
silently ignores a material that fails it; here using one raises instead.

Numbers follow Lua 5.4: integer and float literals both become doubles when
the loader reads them (lua_tonumber), `/` and `^` are float operations, and
the math functions are the C library's."""
from __future__ import annotations

import dataclasses
import math
import os
import re
from typing import Dict, List, Optional, Tuple

from . import _abi as A


class SubsetError(ValueError):
    """The script uses Lua outside the material-file subset."""


class ScriptError(RuntimeError):
    """A Lua run-time error in the script (the reference's lua_pcall would stop
    the script at this point)."""


@dataclasses.dataclass
class MaterialScript:
    eps_inf: float = 1.0
    terms: Dict[str, List[Tuple[float, ...]]] = dataclasses.field(
        default_factory=lambda: {"debye": [], "drude": [], "lorentz": [], "critpoint": []})
    name: str = ""
    description: str = ""
    validity: Tuple[float, float] = (400e-9, 1000e-9)   # Material::reset defaults
    not_fdtd: List[str] = dataclasses.field(default_factory=list)   # models the FDTD cannot run
    error: Optional[str] = None       # the run-time error that stopped the script, if any
    path: str = ""

    def fdtd_compatible(self) -> bool:
        return not self.not_fdtd

    def refusal(self) -> Optional[str]:
        """Why the FDTD cannot use this material (None when it can): a model
        fdtd_compatible rejects, or a script that stopped on a Lua error (the
        reference would go on with the material as it stood at that point,
        which is not what the file describes)."""
        if self.not_fdtd:
            return "not an FDTD model: " + ", ".join(sorted(set(self.not_fdtd)))
        if self.error:
            return "the script stopped on a Lua error: " + self.error
        return None

    def desc(self) -> A.MaterialDesc:
        why = self.refusal()
        if why:
            raise ValueError(f"{os.path.basename(self.path) or 'material'}: {why}")
        t = self.terms
        return A.material_desc(self.eps_inf, debye=t["debye"], drude=t["drude"], lorentz=t["lorentz"],
                               critpoint=t["critpoint"])

    def reset(self):
        """Material::reset (material.cpp:608-640)."""
        self.eps_inf = 1.0
        self.validity = (400e-9, 1000e-9)
        for k in self.terms:
            self.terms[k] = []
        self.not_fdtd = []


# ---- tokens ------------------------------------------------------------------

_TOKEN = re.compile(r"""
    (?P<ws>[ \t\r\n]+)
  | (?P<lcomment>--\[(?P<leq>=*)\[.*?\](?P=leq)\])
  | (?P<comment>--[^\n]*)
  | (?P<lstring>\[(?P<seq>=*)\[.*?\](?P=seq)\])
  | (?P<number>0[xX][0-9a-fA-F]+|(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?)
  | (?P<string>"(?:[^"\\\n]|\\.)*"|'(?:[^'\\\n]|\\.)*')
  | (?P<name>[A-Za-z_][A-Za-z_0-9]*)
  | (?P<op>\.\.|==|~=|<=|>=|//|[-+*/%^#<>=(){}\[\];:,.])
""", re.VERBOSE | re.DOTALL)

_KEYWORDS = {"and", "break", "do", "else", "elseif", "end", "false", "for", "function", "goto", "if", "in",
             "local", "nil", "not", "or", "repeat", "return", "then", "true", "until", "while"}

_ESC = {"n": "\n", "t": "\t", "r": "\r", "a": "\a", "b": "\b", "f": "\f", "v": "\v", "\\": "\\", '"': '"',
        "'": "'", "\n": "\n"}


def _unescape(body: str) -> str:
    out, i = [], 0
    while i < len(body):
        c = body[i]
        if c != "\\":
            out.append(c)
            i += 1
            continue
        n = body[i + 1]
        if n in _ESC:
            out.append(_ESC[n])
            i += 2
        elif n.isdigit():
            m = re.match(r"[0-9]{1,3}", body[i + 1:])
            out.append(chr(int(m.group(0))))
            i += 1 + len(m.group(0))
        else:
            raise SubsetError(f"string escape \\{n} is outside the material-file subset")
    return "".join(out)


def _tokens(src: str):
    pos = 0
    toks = []
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise SubsetError(f"unexpected character {src[pos]!r} at offset {pos}")
        pos = m.end()
        kind = m.lastgroup
        if kind in ("ws", "comment", "lcomment"):
            continue
        text = m.group(kind)
        if kind == "leq" or kind == "seq":
            continue
        if kind == "number":
            v = float(int(text, 16)) if text[:2].lower() == "0x" else float(text)
            toks.append(("num", v))
        elif kind == "string":
            toks.append(("str", _unescape(text[1:-1])))
        elif kind == "lstring":
            body = text[text.index("[", 1) + 1:text.rindex("]", 0, len(text) - 1)]
            toks.append(("str", body[1:] if body.startswith("\n") else body))
        elif kind == "name":
            toks.append(("kw" if text in _KEYWORDS else "name", text))
        else:
            toks.append(("op", text))
    toks.append(("eof", None))
    return toks


# ---- the math library (the C library's functions, as Lua's lmathlib uses them)

_MATH = {
    "pi": math.pi, "huge": math.inf,
    "sqrt": math.sqrt, "exp": math.exp, "sin": math.sin, "cos": math.cos, "tan": math.tan,
    "asin": math.asin, "acos": math.acos, "abs": abs, "floor": lambda x: float(math.floor(x)),
    "ceil": lambda x: float(math.ceil(x)), "fmod": math.fmod,
    "log": lambda x, b=None: math.log(x) if b is None else (math.log2(x) if b == 2 else
                                                            (math.log10(x) if b == 10 else math.log(x) / math.log(b))),
    "atan": lambda y, x=1.0: math.atan2(y, x),
    "max": lambda *a: max(a), "min": lambda *a: min(a),
}


# ---- parser / evaluator ------------------------------------------------------

class _Run:
    BINARY = {"+": 5, "-": 5, "*": 6, "/": 6, "%": 6, "..": 4}   # Lua 5.4 priorities ("^" handled apart)

    def __init__(self, toks, mat: MaterialScript, base_dir: str, depth: int):
        self.t = toks
        self.i = 0
        self.mat = mat
        self.env: Dict[str, object] = {"math": _MATH}
        self.base = base_dir
        self.depth = depth

    def peek(self, k=0):
        return self.t[self.i + k]

    def take(self, kind=None, text=None):
        tok = self.t[self.i]
        if (kind and tok[0] != kind) or (text is not None and tok[1] != text):
            raise SubsetError(f"expected {text or kind}, found {tok[1]!r}")
        self.i += 1
        return tok

    # statements: `[local] name = expr`, `name(args)`, `name "str"`, `;`
    def run(self):
        while self.peek()[0] != "eof":
            tok = self.peek()
            if tok == ("op", ";"):
                self.i += 1
                continue
            if tok == ("kw", "local"):
                self.i += 1
                tok = self.peek()
            if tok[0] != "name":
                raise SubsetError(f"statement starting with {tok[1]!r} is outside the material-file subset")
            name = self.take("name")[1]
            nxt = self.peek()
            if nxt == ("op", "="):
                self.i += 1
                self.env[name] = self.expr()
            elif nxt == ("op", "(") or nxt[0] == "str":
                args = self.call_args()
                self.call(name, args)
            else:
                raise SubsetError(f"statement `{name} {nxt[1]}` is outside the material-file subset")

    def call_args(self):
        if self.peek()[0] == "str":
            return [self.take()[1]]
        self.take("op", "(")
        args = []
        if self.peek() != ("op", ")"):
            args.append(self.expr())
            while self.peek() == ("op", ","):
                self.i += 1
                args.append(self.expr())
        self.take("op", ")")
        return args

    def expr(self, limit=0):
        left = self.unary()
        while True:
            tok = self.peek()
            if tok[0] != "op" or tok[1] not in self.BINARY or self.BINARY[tok[1]] <= limit:
                return left
            op = tok[1]
            self.i += 1
            # ".." is right associative
            right = self.expr(self.BINARY[op] - (1 if op == ".." else 0))
            left = self._binary(op, left, right)

    def unary(self):
        tok = self.peek()
        if tok == ("op", "-"):
            self.i += 1
            v = self.unary()
            return -self._num(v)
        return self.power()

    def power(self):
        base = self.primary()
        if self.peek() == ("op", "^"):
            self.i += 1
            exp = self.unary()   # right associative, binds tighter than unary minus on its left
            return math.pow(self._num(base), self._num(exp))
        return base

    def primary(self):
        tok = self.take()
        if tok[0] in ("num", "str"):
            return tok[1]
        if tok == ("op", "("):
            v = self.expr()
            self.take("op", ")")
            return v
        if tok == ("op", "{"):
            # list constructor {e1, e2, ...} (the tabulated-data files' vectors)
            items = []
            while self.peek() != ("op", "}"):
                items.append(self.expr())
                if self.peek() in (("op", ","), ("op", ";")):
                    self.i += 1
                elif self.peek() != ("op", "}"):
                    raise SubsetError("table constructor outside the material-file subset")
            self.take("op", "}")
            return items
        if tok[0] == "name":
            v = self.env.get(tok[1])
            while self.peek() == ("op", "."):
                self.i += 1
                field = self.take("name")[1]
                if not isinstance(v, dict) or field not in v:
                    raise ScriptError(f"attempt to index field '{field}'")
                v = v[field]
            if self.peek() == ("op", "(") or self.peek()[0] == "str":
                args = self.call_args()
                if callable(v):
                    return float(v(*[self._num(a) for a in args]))
                raise SubsetError(f"call of {tok[1]!r} inside an expression is outside the material-file subset")
            if v is None:
                raise ScriptError(f"attempt to use the nil value '{tok[1]}'")
            return v
        raise SubsetError(f"expression starting with {tok[1]!r} is outside the material-file subset")

    @staticmethod
    def _num(v):
        if isinstance(v, float):
            return v
        if isinstance(v, str):
            try:
                return float(v)   # Lua coerces numeric strings in arithmetic
            except ValueError:
                pass
        raise ScriptError(f"attempt to perform arithmetic on a {type(v).__name__} value")

    def _binary(self, op, a, b):
        if op == "..":
            def s(v):
                if isinstance(v, float):
                    return repr(int(v)) if v.is_integer() and abs(v) < 2 ** 53 else repr(v)
                return v
            return s(a) + s(b)
        x, y = self._num(a), self._num(b)
        if op == "+":
            return x + y
        if op == "-":
            return x - y
        if op == "*":
            return x * y
        if op == "/":
            return x / y if y != 0 else (math.copysign(math.inf, x) * math.copysign(1.0, y) if x != 0 else math.nan)
        return x - math.floor(x / y) * y   # "%"

    # the loader's functions (lua_material.cpp:100-380)
    def call(self, name, args):
        m = self.mat

        def num(k):
            # lua_tonumber: the number, a numeric string's value, else 0
            if k >= len(args):
                return 0.0
            v = args[k]
            if isinstance(v, float):
                return v
            try:
                return float(v)
            except (TypeError, ValueError):
                return 0.0

        if name in ("epsilon_infty", "epsilon_infinity"):
            m.eps_inf = num(0)
        elif name in ("index_infty", "index_infinity", "refractive_index"):
            n = num(0)
            m.eps_inf = n * n
        elif name == "add_debye":
            m.terms["debye"].append((num(0), num(1)))
        elif name == "add_drude":
            m.terms["drude"].append((num(0), num(1)))
        elif name == "add_lorentz":
            m.terms["lorentz"].append((num(0), num(1), num(2)))
        elif name == "add_crit_point":
            m.terms["critpoint"].append((num(0), num(1), num(2), num(3)))
        elif name == "add_cauchy":
            m.not_fdtd.append("Cauchy")
        elif name == "add_sellmeier":
            m.not_fdtd.append("Sellmeier")
        elif name in ("add_data_index", "add_data_epsilon"):
            m.not_fdtd.append("tabulated data (spline)")
        elif name in ("add_effective_component", "effective_host", "effective_type"):
            m.not_fdtd.append("effective medium")
        elif name == "name":
            m.name = str(args[0]) if args else ""
        elif name == "description":
            m.description = str(args[0]) if args else ""
        elif name == "validity_range":
            m.validity = (num(0), num(1))
        elif name == "load_script":
            if self.depth > 8:
                raise ScriptError("load_script nested too deeply")
            path = str(args[0]) if args else ""
            if not os.path.isabs(path):
                path = os.path.join(self.base, path)
            _load_into(m, path, self.depth + 1)
        elif name in _MATH and callable(_MATH[name]):
            pass
        else:
            raise ScriptError(f"attempt to call a nil value (global '{name}')")


def _load_into(mat: MaterialScript, path: str, depth: int = 0):
    """Loader::load (lua_material.cpp:466-497): reset, then run the script;
    a run-time error stops it there (lua_pcall), and is recorded."""
    if not os.path.isfile(path):
        raise FileNotFoundError(f"material file {path!r} not found")
    with open(path, encoding="utf-8", errors="replace") as f:
        src = f.read()
    mat.reset()
    mat.path = path
    toks = _tokens(src)   # syntax outside the subset raises before anything runs, as luaL_loadfile would
    try:
        _Run(toks, mat, os.path.dirname(path), depth).run()
    except ScriptError as e:
        mat.error = str(e)


def load_file(path: str) -> MaterialScript:
    """Reads one material file. Raises SubsetError for Lua outside the subset
    the library's files use; a Lua run-time error stops the script (as in the
    reference) and is kept in `.error`; `.refusal()` says why the FDTD cannot
    use the material, if it cannot."""
    m = MaterialScript()
    _load_into(m, path)
    return m
