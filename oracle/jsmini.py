"""TEST INFRASTRUCTURE ONLY: a small interpreter for the JavaScript subset that the
reference's tree-build modules are written in, so that tests can run the
reference's own source text (src/physics/mortonTree.js, src/physics/bhWorker.js)
and compare its outputs with the C++ oracle and with the CUDA path. Nothing in
the product imports it.

It parses an ES module, translates it to Python source that keeps the
JavaScript semantics the subset relies on, and runs that:
  * numbers are IEEE doubles (Python floats; integer-valued results of integer
    operands stay Python ints, exact below 2^53);
  * `|`, `&`, `^`, `~`, `<<`, `>>` act on ToInt32, `>>>` on ToUint32 (ToInt32
    truncates toward zero and maps NaN and +-Infinity to 0);
  * `/` and `%` give Infinity / NaN instead of raising; unary minus of 0 is -0;
    `Math.min` / `Math.max` propagate NaN; `Number.isFinite`;
  * typed arrays (Float32Array, Float64Array, Int32Array, Uint32Array,
    Uint8Array, ...) over shared ArrayBuffers: stores round to float32 or wrap
    modulo 2^32 as the JS engine does, out-of-range reads give undefined,
    out-of-range writes are dropped; subarray / set / fill / slice;
  * arrays (push, length, live for-of iteration), object literals (shorthand
    properties too), classes with constructors, methods and getters, `new`,
    closures over module variables, arrow functions, default parameters, `??`,
    `&&`, `||` and conditions with JavaScript truthiness;
  * `let` / `const` block scoping (each declaration gets its own Python name),
    hoisting of a block's declarations, ES imports between modules.
The subset has no regular-expression literals, labels, generators, exceptions
or prototype manipulation; a construct outside it raises JsSyntaxError or
JsRuntimeError instead of being guessed at.
"""
from __future__ import annotations

import math
import os
import re
import struct

__all__ = ["load_module", "run_source", "TA", "JSObject", "JSArray", "JSArrayBuffer", "JSFunction",
           "to_numpy", "from_numpy", "construct", "call_value", "call_method", "get_prop", "NULL",
           "JsSyntaxError", "JsRuntimeError"]


class JsSyntaxError(SyntaxError):
    pass


class JsRuntimeError(RuntimeError):
    pass


# ---------------------------------------------------------------------------- lexer

_TOKEN = re.compile(r"""
 (?P<ws>[ \t\r\n]+)
|(?P<lc>//[^\n]*)
|(?P<bc>/\*.*?\*/)
|(?P<num>0[xX][0-9a-fA-F]+|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)
|(?P<str>'(?:[^'\\\n]|\\.)*'|"(?:[^"\\\n]|\\.)*")
|(?P<id>[A-Za-z_$][A-Za-z0-9_$]*)
|(?P<op>>>>=|>>>|===|!==|\?\?=|&&=|\|\|=|\.\.\.|<<=|>>=|\*\*=|=>|==|!=|<=|>=|&&|\|\||\?\?|\+\+|--|\+=|-=|\*=|/=|%=|&=|\|=|\^=|<<|>>|\*\*|[{}()\[\];,.<>+\-*/%&|^!~?:=])
""", re.S | re.X)

_ESCAPES = {"n": "\n", "t": "\t", "r": "\r", "0": "\0", "\\": "\\", "'": "'", '"': '"', "b": "\b",
            "f": "\f", "v": "\v"}


def _unescape(s):
    body, out, i = s[1:-1], [], 0
    while i < len(body):
        c = body[i]
        if c == "\\" and i + 1 < len(body):
            n = body[i + 1]
            if n in _ESCAPES:
                out.append(_ESCAPES[n])
                i += 2
            elif n == "x":
                out.append(chr(int(body[i + 2:i + 4], 16)))
                i += 4
            elif n == "u":
                out.append(chr(int(body[i + 2:i + 6], 16)))
                i += 6
            else:
                out.append(n)
                i += 2
            continue
        out.append(c)
        i += 1
    return "".join(out)


def tokenize(src):
    """Tokens (kind, value, line, newline_before)."""
    toks, pos, line, nl = [], 0, 1, False
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise JsSyntaxError(f"line {line}: unexpected character {src[pos]!r}")
        kind, text = m.lastgroup, m.group(m.lastgroup)
        if kind in ("ws", "lc", "bc"):
            nl = nl or "\n" in text
        elif kind == "num":
            if text[:2] in ("0x", "0X"):
                val = int(text, 16)
            elif re.fullmatch(r"\d+", text):
                val = int(text)
            else:
                val = float(text)
            toks.append(("num", val, line, nl))
            nl = False
        elif kind == "str":
            toks.append(("str", _unescape(text), line, nl))
            nl = False
        else:
            toks.append((kind, text, line, nl))
            nl = False
        line += text.count("\n")
        pos = m.end()
    toks.append(("eof", None, line, True))
    return toks


# ---------------------------------------------------------------------------- parser

_BINARY_PREC = {
    "??": 1, "||": 2, "&&": 3, "|": 4, "^": 5, "&": 6,
    "==": 7, "!=": 7, "===": 7, "!==": 7, "<": 8, ">": 8, "<=": 8, ">=": 8,
    "<<": 9, ">>": 9, ">>>": 9, "+": 10, "-": 10, "*": 11, "/": 11, "%": 11, "**": 12,
}
_ASSIGN_OPS = {"=", "+=", "-=", "*=", "/=", "%=", "<<=", ">>=", ">>>=", "&=", "|=", "^=", "**=",
               "??=", "&&=", "||="}
_OUTSIDE = {"switch", "try", "throw", "with", "yield", "async", "await", "delete", "instanceof", "in"}


class Parser:
    """Recursive-descent parser of the subset into tuples ("kind", ...)."""

    def __init__(self, src):
        self.t = tokenize(src)
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k]

    def at(self, kind, val=None, k=0):
        tok = self.t[self.i + k]
        return tok[0] == kind and (val is None or tok[1] == val)

    def at_op(self, val, k=0):
        return self.at("op", val, k)

    def at_kw(self, val, k=0):
        return self.at("id", val, k)

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def expect_op(self, val):
        tok = self.next()
        if tok[0] != "op" or tok[1] != val:
            raise JsSyntaxError(f"line {tok[2]}: expected {val!r}, got {tok[1]!r}")

    def expect_id(self):
        tok = self.next()
        if tok[0] != "id":
            raise JsSyntaxError(f"line {tok[2]}: expected an identifier, got {tok[1]!r}")
        return tok[1]

    def semi(self):
        if self.at_op(";"):
            self.next()
            return
        tok = self.peek()
        if tok[0] == "eof" or tok[3] or self.at_op("}"):
            return  # automatic semicolon insertion
        raise JsSyntaxError(f"line {tok[2]}: expected ';', got {tok[1]!r}")

    def program(self):
        body = []
        while not self.at("eof"):
            body.append(self.statement(top=True))
        return body

    def statement(self, top=False):
        tok = self.peek()
        if tok[0] == "op" and tok[1] == "{":
            return ("block", self.block())
        if tok[0] == "op" and tok[1] == ";":
            self.next()
            return ("empty",)
        if tok[0] == "id":
            v = tok[1]
            if v == "export" and top:
                self.next()
                if self.at_kw("default"):
                    raise JsSyntaxError(f"line {tok[2]}: export default is outside the subset")
                return ("export", self.statement(top=True))
            if v == "import" and top:
                return self.import_decl()
            if v in ("const", "let", "var"):
                d = self.var_decl()
                self.semi()
                return d
            if v == "function":
                self.next()
                name = self.expect_id()
                params, body = self.function_rest()
                return ("funcdecl", name, params, body)
            if v == "class":
                return self.class_decl()
            if v == "if":
                self.next()
                self.expect_op("(")
                test = self.expression()
                self.expect_op(")")
                cons = self.statement()
                alt = None
                if self.at_kw("else"):
                    self.next()
                    alt = self.statement()
                return ("if", test, cons, alt)
            if v == "for":
                return self.for_stmt()
            if v == "while":
                self.next()
                self.expect_op("(")
                test = self.expression()
                self.expect_op(")")
                return ("while", test, self.statement())
            if v == "do":
                self.next()
                body = self.statement()
                if not self.at_kw("while"):
                    raise JsSyntaxError("expected while after do")
                self.next()
                self.expect_op("(")
                test = self.expression()
                self.expect_op(")")
                self.semi()
                return ("dowhile", body, test)
            if v == "return":
                self.next()
                e = None
                if not (self.at_op(";") or self.at_op("}") or self.peek()[3] or self.at("eof")):
                    e = self.expression()
                self.semi()
                return ("return", e)
            if v in ("break", "continue"):
                self.next()
                if self.at("id") and not self.peek()[3]:
                    raise JsSyntaxError(f"line {tok[2]}: labels are outside the subset")
                self.semi()
                return (v,)
            if v in _OUTSIDE:
                raise JsSyntaxError(f"line {tok[2]}: '{v}' is outside the subset")
        e = self.expression()
        self.semi()
        return ("expr", e)

    def block(self):
        self.expect_op("{")
        body = []
        while not self.at_op("}"):
            body.append(self.statement())
        self.next()
        return body

    def import_decl(self):
        self.next()
        names = []
        self.expect_op("{")
        while not self.at_op("}"):
            imported = self.expect_id()
            local = imported
            if self.at_kw("as"):
                self.next()
                local = self.expect_id()
            names.append((imported, local))
            if self.at_op(","):
                self.next()
        self.next()
        if not self.at_kw("from"):
            raise JsSyntaxError("expected from")
        self.next()
        src = self.next()
        if src[0] != "str":
            raise JsSyntaxError("expected a module path")
        self.semi()
        return ("import", names, src[1])

    def var_decl(self):
        kind = self.next()[1]
        decls = []
        while True:
            name = self.expect_id()
            init = None
            if self.at_op("="):
                self.next()
                init = self.assign_expr()
            decls.append((name, init))
            if not self.at_op(","):
                return ("var", kind, decls)
            self.next()

    def for_stmt(self):
        self.next()
        self.expect_op("(")
        init = None
        if self.at_kw("const") or self.at_kw("let") or self.at_kw("var"):
            if self.at("id", None, 1) and self.at_kw("of", 2):
                kind = self.next()[1]
                name = self.expect_id()
                self.next()
                it = self.assign_expr()
                self.expect_op(")")
                return ("forof", kind, name, it, self.statement())
            if self.at("id", None, 1) and self.at_kw("in", 2):
                raise JsSyntaxError("for-in is outside the subset")
            init = self.var_decl()
        elif not self.at_op(";"):
            init = ("expr", self.expression())
        self.expect_op(";")
        test = None if self.at_op(";") else self.expression()
        self.expect_op(";")
        update = None if self.at_op(")") else self.expression()
        self.expect_op(")")
        return ("for", init, test, update, self.statement())

    def class_decl(self):
        self.next()
        name = self.expect_id()
        if self.at_kw("extends"):
            raise JsSyntaxError("class inheritance is outside the subset")
        self.expect_op("{")
        members = []
        while not self.at_op("}"):
            if self.at_op(";"):
                self.next()
                continue
            kind = "method"
            if (self.at_kw("get") or self.at_kw("set") or self.at_kw("static")) and self.at("id", None, 1):
                kind = self.next()[1]
            mname = self.expect_id()
            params, body = self.function_rest()
            if mname == "constructor" and kind == "method":
                kind = "ctor"
            members.append((kind, mname, params, body))
        self.next()
        return ("class", name, members)

    def function_rest(self):
        self.expect_op("(")
        params = self.params_until(")")
        return params, self.block()

    def params_until(self, close):
        params = []
        while not self.at_op(close):
            if self.at_op("...") or self.at_op("{") or self.at_op("["):
                raise JsSyntaxError("rest and destructured parameters are outside the subset")
            name = self.expect_id()
            default = None
            if self.at_op("="):
                self.next()
                default = self.assign_expr()
            params.append((name, default))
            if self.at_op(","):
                self.next()
        self.next()
        return params

    def expression(self):
        e = self.assign_expr()
        if not self.at_op(","):
            return e
        seq = [e]
        while self.at_op(","):
            self.next()
            seq.append(self.assign_expr())
        return ("seq", seq)

    def arrow_ahead(self):
        if self.at("id") and self.at_op("=>", 1):
            return True
        if not self.at_op("("):
            return False
        depth, k = 0, 0
        while True:
            tok = self.peek(k)
            if tok[0] == "eof":
                return False
            if tok[0] == "op" and tok[1] in ("(", "[", "{"):
                depth += 1
            elif tok[0] == "op" and tok[1] in (")", "]", "}"):
                depth -= 1
                if depth == 0:
                    return self.at_op("=>", k + 1)
            k += 1

    def arrow(self):
        if self.at("id"):
            params = [(self.next()[1], None)]
        else:
            self.next()
            params = self.params_until(")")
        self.expect_op("=>")
        body = self.block() if self.at_op("{") else [("return", self.assign_expr())]
        return ("funcexpr", None, params, body, True)

    def assign_expr(self):
        if self.arrow_ahead():
            return self.arrow()
        left = self.cond_expr()
        if self.at("op") and self.peek()[1] in _ASSIGN_OPS:
            op = self.next()[1]
            if left[0] not in ("id", "member", "index"):
                raise JsSyntaxError("invalid assignment target")
            return ("assign", op, left, self.assign_expr())
        return left

    def cond_expr(self):
        test = self.binary(0)
        if not self.at_op("?"):
            return test
        self.next()
        a = self.assign_expr()
        self.expect_op(":")
        return ("cond", test, a, self.assign_expr())

    def binary(self, min_prec):
        left = self.unary()
        while True:
            tok = self.peek()
            op = tok[1] if tok[0] == "op" else None
            prec = _BINARY_PREC.get(op) if op else None
            if prec is None or prec <= min_prec:
                return left
            self.next()
            right = self.binary(prec - 1 if op == "**" else prec)
            left = ("logic" if op in ("&&", "||", "??") else "bin", op, left, right)

    def unary(self):
        tok = self.peek()
        if tok[0] == "op" and tok[1] in ("!", "-", "+", "~"):
            self.next()
            return ("unary", tok[1], self.unary())
        if tok[0] == "op" and tok[1] in ("++", "--"):
            self.next()
            return ("update", tok[1], True, self.unary())
        if tok[0] == "id" and tok[1] in ("typeof", "void"):
            self.next()
            return ("unary", tok[1], self.unary())
        e = self.call_member()
        tok = self.peek()
        if tok[0] == "op" and tok[1] in ("++", "--") and not tok[3]:
            self.next()
            return ("update", tok[1], False, e)
        return e

    def call_member(self):
        if self.at_kw("new"):
            self.next()
            callee = self.member_chain(self.primary(), calls=False)
            args = self.arguments() if self.at_op("(") else []
            e = ("new", callee, args)
        else:
            e = self.primary()
        return self.member_chain(e, calls=True)

    def member_chain(self, e, calls):
        while True:
            if self.at_op("."):
                self.next()
                e = ("member", e, self.expect_id())
            elif self.at_op("["):
                self.next()
                k = self.expression()
                self.expect_op("]")
                e = ("index", e, k)
            elif calls and self.at_op("("):
                e = ("call", e, self.arguments())
            else:
                return e

    def arguments(self):
        self.expect_op("(")
        args = []
        while not self.at_op(")"):
            if self.at_op("..."):
                raise JsSyntaxError("spread arguments are outside the subset")
            args.append(self.assign_expr())
            if self.at_op(","):
                self.next()
        self.next()
        return args

    def primary(self):
        tok = self.next()
        kind, v = tok[0], tok[1]
        if kind == "num":
            return ("num", v)
        if kind == "str":
            return ("str", v)
        if kind == "id":
            if v == "true":
                return ("bool", True)
            if v == "false":
                return ("bool", False)
            if v == "null":
                return ("null",)
            if v == "this":
                return ("this",)
            if v == "function":
                name = self.expect_id() if self.at("id") else None
                params, body = self.function_rest()
                return ("funcexpr", name, params, body, False)
            if v in _OUTSIDE:
                raise JsSyntaxError(f"line {tok[2]}: '{v}' is outside the subset")
            return ("id", v)
        if kind == "op" and v == "(":
            e = self.expression()
            self.expect_op(")")
            return e
        if kind == "op" and v == "[":
            elems = []
            while not self.at_op("]"):
                if self.at_op("...") or self.at_op(","):
                    raise JsSyntaxError("spread elements and holes are outside the subset")
                elems.append(self.assign_expr())
                if self.at_op(","):
                    self.next()
            self.next()
            return ("array", elems)
        if kind == "op" and v == "{":
            props = []
            while not self.at_op("}"):
                ktok = self.next()
                if ktok[0] not in ("id", "str", "num"):
                    raise JsSyntaxError(f"line {ktok[2]}: bad property key {ktok[1]!r}")
                key = str(ktok[1])
                if self.at_op(":"):
                    self.next()
                    props.append((key, self.assign_expr()))
                elif self.at_op("("):
                    params, body = self.function_rest()
                    props.append((key, ("funcexpr", key, params, body, False)))
                else:
                    props.append((key, ("id", key)))   # shorthand property
                if self.at_op(","):
                    self.next()
            self.next()
            return ("object", props)
        raise JsSyntaxError(f"line {tok[2]}: unexpected {v!r}")


# ---------------------------------------------------------------------------- values


class _Null:
    __slots__ = ()

    def __repr__(self):
        return "null"

    def __bool__(self):
        return False


NULL = _Null()   # JavaScript null; undefined is Python None


class JSArrayBuffer:
    __slots__ = ("data",)

    def __init__(self, n_or_bytes):
        self.data = n_or_bytes if isinstance(n_or_bytes, bytearray) else bytearray(n_or_bytes)


_TA_KINDS = {"Float32Array": ("f", 4), "Float64Array": ("d", 8), "Int32Array": ("i", 4),
             "Uint32Array": ("I", 4), "Uint8Array": ("B", 1), "Int8Array": ("b", 1),
             "Int16Array": ("h", 2), "Uint16Array": ("H", 2)}


def to_number(v):
    t = type(v)
    if t is int or t is float:
        return v
    if t is bool:
        return 1 if v else 0
    if v is None:
        return math.nan
    if v is NULL:
        return 0
    if t is str:
        s = v.strip()
        if not s:
            return 0
        try:
            return int(s, 16) if re.fullmatch(r"0[xX][0-9a-fA-F]+", s) else (
                int(s) if re.fullmatch(r"[+-]?\d+", s) else float(s))
        except ValueError:
            return math.nan
    return math.nan


def to_int32(v):
    if type(v) is int:
        if -2147483648 <= v <= 2147483647:
            return v
    else:
        v = to_number(v)
        if type(v) is float:
            if v != v or v in (math.inf, -math.inf):
                return 0
            v = int(v)   # truncation toward zero
    v &= 0xFFFFFFFF
    return v - 0x100000000 if v >= 0x80000000 else v


def to_uint32(v):
    if type(v) is int:
        if 0 <= v <= 0xFFFFFFFF:
            return v
    else:
        v = to_number(v)
        if type(v) is float:
            if v != v or v in (math.inf, -math.inf):
                return 0
            v = int(v)
    return v & 0xFFFFFFFF


def _int_store(bits, signed):
    mask = (1 << bits) - 1

    def conv(v):
        if type(v) is not int:
            v = to_number(v)
            if type(v) is float:
                if v != v or v in (math.inf, -math.inf):
                    return 0
                v = int(v)
        v &= mask
        return v - (1 << bits) if signed and v >= 1 << (bits - 1) else v
    return conv


def _float_store(v):
    return v if type(v) is float else float(to_number(v))


_CONV = {"f": _float_store, "d": _float_store, "i": to_int32, "I": to_uint32,
         "B": _int_store(8, False), "b": _int_store(8, True), "h": _int_store(16, True),
         "H": _int_store(16, False)}


class TA:
    """A typed-array view (kind, byte offset, length) over a JSArrayBuffer. Stores
    through a memoryview of format 'f' round a double to float32 exactly as
    Float32Array does (round to nearest even, overflow to infinity)."""

    __slots__ = ("kind", "fmt", "size", "buffer", "offset", "n", "mv", "conv")

    def __init__(self, kind, buffer, offset, n):
        self.kind = kind
        self.fmt, self.size = _TA_KINDS[kind]
        self.buffer, self.offset, self.n = buffer, offset, n
        self.mv = memoryview(buffer.data)[offset:offset + n * self.size].cast(self.fmt)
        self.conv = _CONV[self.fmt]

    def __len__(self):
        return self.n

    def __bool__(self):
        return True


class JSArray(list):
    __slots__ = ()

    def __bool__(self):
        return True

    __hash__ = object.__hash__

    def __eq__(self, other):
        return self is other


class JSClass:
    __slots__ = ("name", "ctor", "methods", "getters", "setters", "statics")

    def __init__(self, name, ctor, methods, getters, setters, statics):
        self.name, self.ctor, self.methods = name, ctor, methods
        self.getters, self.setters, self.statics = getters, setters, statics


class JSObject:
    __slots__ = ("props", "proto")

    def __init__(self, props=None, proto=None):
        self.props = {} if props is None else props
        self.proto = proto

    def __repr__(self):
        return f"JSObject({self.props!r})"


class JSFunction:
    """A function value: a Python callable taking (this, *args)."""

    __slots__ = ("fn", "name")

    def __init__(self, fn, name=""):
        self.fn, self.name = fn, name


class Namespace:
    """A built-in namespace object (Math, Number, console)."""

    def __init__(self, name, **members):
        self.name, self.members = name, members


def truthy(v):
    t = type(v)
    if t is bool:
        return v
    if t is int:
        return v != 0
    if t is float:
        return v == v and v != 0.0
    if t is str:
        return len(v) > 0
    return not (v is None or v is NULL)


def to_string(v):
    if v is None:
        return "undefined"
    if v is NULL:
        return "null"
    t = type(v)
    if t is bool:
        return "true" if v else "false"
    if t is int:
        return str(v)
    if t is float:
        if v != v:
            return "NaN"
        if v in (math.inf, -math.inf):
            return "Infinity" if v > 0 else "-Infinity"
        return str(int(v)) if v.is_integer() and abs(v) < 1e21 else repr(v)
    if t is str:
        return v
    if t is JSArray:
        return ",".join("" if x is None or x is NULL else to_string(x) for x in v)
    return "[object Object]"


# ---------------------------------------------------------------------------- operators


def op_add(a, b):
    ta, tb = type(a), type(b)
    if (ta is int or ta is float) and (tb is int or tb is float):
        return a + b
    if ta is str or tb is str:
        return to_string(a) + to_string(b)
    return to_number(a) + to_number(b)


def op_sub(a, b):
    return to_number(a) - to_number(b)


def op_mul(a, b):
    return to_number(a) * to_number(b)


def op_div(a, b):
    a, b = to_number(a), to_number(b)
    try:
        return a / b
    except ZeroDivisionError:
        if a != a or a == 0:
            return math.nan
        return -math.inf if (a < 0) != (math.copysign(1.0, b) < 0) else math.inf


def op_mod(a, b):
    a, b = to_number(a), to_number(b)
    if b == 0 or a != a or b != b or a in (math.inf, -math.inf):
        return math.nan
    if type(a) is int and type(b) is int:
        r = abs(a) % abs(b)
        return (-r if r else -0.0) if a < 0 else r
    return math.fmod(a, b)


def op_neg(a):
    a = to_number(a)
    return -0.0 if type(a) is int and a == 0 else -a


def op_pow(a, b):
    try:
        return float(to_number(a)) ** float(to_number(b))
    except (OverflowError, ZeroDivisionError):
        return math.inf


def op_shl(a, b):
    return to_int32(to_int32(a) << (to_uint32(b) & 31))


def op_sar(a, b):
    return to_int32(a) >> (to_uint32(b) & 31)


def op_shr(a, b):
    return to_uint32(a) >> (to_uint32(b) & 31)


def op_or(a, b):
    return to_int32(to_int32(a) | to_int32(b))


def op_and(a, b):
    return to_int32(to_int32(a) & to_int32(b))


def op_xor(a, b):
    return to_int32(to_int32(a) ^ to_int32(b))


def op_not(a):
    return to_int32(~to_int32(a))


def strict_eq(a, b):
    ta, tb = type(a), type(b)
    if (ta is int or ta is float) and (tb is int or tb is float):
        return a == b
    if ta is bool or tb is bool or ta is str or tb is str:
        return ta is tb and a == b
    return a is b


def loose_eq(a, b):
    if (a is None or a is NULL) or (b is None or b is NULL):
        return (a is None or a is NULL) and (b is None or b is NULL)
    prim = (int, float, bool, str)
    if type(a) in prim and type(b) in prim:
        if type(a) is str and type(b) is str:
            return a == b
        return to_number(a) == to_number(b)
    return a is b


def op_lt(a, b):
    if type(a) is str and type(b) is str:
        return a < b
    return to_number(a) < to_number(b)


def op_gt(a, b):
    return op_lt(b, a)


def op_le(a, b):
    if type(a) is str and type(b) is str:
        return a <= b
    return to_number(a) <= to_number(b)


def op_ge(a, b):
    if type(a) is str and type(b) is str:
        return a >= b
    return to_number(a) >= to_number(b)


def typeof(v):
    if v is None:
        return "undefined"
    t = type(v)
    if t is bool:
        return "boolean"
    if t is int or t is float:
        return "number"
    if t is str:
        return "string"
    if t in (JSFunction, JSClass) or (callable(v) and t not in (TA, JSObject, JSArray)):
        return "function"
    return "object"


# ---------------------------------------------------------------------------- properties


def _index_key(k):
    t = type(k)
    if t is int:
        return k
    if t is float and k.is_integer():
        return int(k)
    if t is str and re.fullmatch(r"0|[1-9]\d*", k):
        return int(k)
    return to_string(k)


def _ta_prop(o, name):
    if name == "length":
        return o.n
    if name == "buffer":
        return o.buffer
    if name == "byteOffset":
        return o.offset
    if name == "byteLength":
        return o.n * o.size
    if name == "BYTES_PER_ELEMENT":
        return o.size
    return None


def get_prop(o, name):
    t = type(o)
    if t is JSObject:
        d = o.props
        if name in d:
            return d[name]
        c = o.proto
        if c is not None:
            if name in c.getters:
                return c.getters[name](o)
            return c.methods.get(name)
        return None
    if t is TA:
        return _ta_prop(o, name)
    if t is JSArray or t is str:
        return len(o) if name == "length" else None
    if t is JSArrayBuffer:
        return len(o.data) if name == "byteLength" else None
    if t is Namespace:
        return o.members.get(name)
    if t is JSClass:
        return o.statics.get(name)
    if o is None or o is NULL:
        raise JsRuntimeError(f"TypeError: cannot read property {name!r} of {to_string(o)}")
    return None


def get_key(o, k):
    t = type(o)
    if t is TA:
        if type(k) is not int:
            k = _index_key(k)
            if type(k) is not int:
                return _ta_prop(o, k)
        return o.mv[k] if 0 <= k < o.n else None
    if t is JSArray:
        if type(k) is not int:
            k = _index_key(k)
            if type(k) is not int:
                return get_prop(o, k)
        return o[k] if 0 <= k < len(o) else None
    k = _index_key(k)
    return get_prop(o, str(k) if type(k) is int else k)


def set_prop(o, name, v):
    t = type(o)
    if t is JSObject:
        c = o.proto
        if c is not None and name in c.setters:
            c.setters[name](o, v)
        else:
            o.props[name] = v
        return v
    if t is JSArray and name == "length":
        n = to_uint32(v)
        del o[n:]
        o.extend([None] * (n - len(o)))
        return v
    if o is None or o is NULL:
        raise JsRuntimeError(f"TypeError: cannot set property {name!r} of {to_string(o)}")
    raise JsRuntimeError(f"setting {name!r} on a {t.__name__} is outside the subset")


def set_key(o, k, v):
    t = type(o)
    if t is TA:
        if type(k) is not int:
            k = _index_key(k)
        if type(k) is int and 0 <= k < o.n:
            o.mv[k] = o.conv(v)
        return v
    if t is JSArray:
        if type(k) is not int:
            k = _index_key(k)
            if type(k) is not int:
                return set_prop(o, k, v)
        if k < len(o):
            o[k] = v
        else:
            o.extend([None] * (k - len(o)))
            o.append(v)
        return v
    k = _index_key(k)
    return set_prop(o, str(k) if type(k) is int else k, v)


def aug_prop(o, k, fn, v):
    r = fn(get_prop(o, k), v)
    set_prop(o, k, r)
    return r


def aug_prop_lazy(o, k, fn, thunk):
    old = get_prop(o, k)
    r = fn(old, thunk())
    set_prop(o, k, r)
    return r


def aug_key(o, k, fn, v):
    r = fn(get_key(o, k), v)
    set_key(o, k, r)
    return r


def aug_key_lazy(o, k, fn, thunk):
    old = get_key(o, k)
    r = fn(old, thunk())
    set_key(o, k, r)
    return r


def upd_prop(o, k, d, prefix):
    old = to_number(get_prop(o, k))
    set_prop(o, k, old + d)
    return old + d if prefix else old


def upd_key(o, k, d, prefix):
    if type(o) is TA and type(k) is int and 0 <= k < o.n:
        old = o.mv[k]
        o.mv[k] = o.conv(old + d)
        return old + d if prefix else old
    old = to_number(get_key(o, k))
    set_key(o, k, old + d)
    return old + d if prefix else old


def range_stop(b, inclusive):
    """Exclusive Python range end of a counted loop `i < b` / `i <= b` from 0 up."""
    b = to_number(b)
    if type(b) is float:
        if b != b:
            return 0
        if b in (math.inf, -math.inf):
            raise JsRuntimeError("an unbounded counted loop is outside the subset")
        return math.floor(b) + 1 if inclusive or not b.is_integer() else int(b)
    return b + 1 if inclusive else b


def iterate(v):
    t = type(v)
    if t is JSArray:
        return v      # live: elements pushed during the loop are visited, as in JS
    if t is TA:
        return (v.mv[i] for i in range(v.n))
    if t is str:
        return iter(v)
    raise JsRuntimeError(f"TypeError: {to_string(v)} is not iterable")


# ---------------------------------------------------------------------------- built-ins


def _rel_index(v, n):
    v = to_number(v)
    if v != v:
        return 0
    if v in (math.inf, -math.inf):
        return n if v > 0 else 0
    v = int(v)
    return max(0, n + v) if v < 0 else min(v, n)


def _new_ta(kind, args):
    fmt, size = _TA_KINDS[kind]
    a0 = args[0] if args else None
    t = type(a0)
    if a0 is None:
        return TA(kind, JSArrayBuffer(0), 0, 0)
    if t is int or t is float:
        n = to_uint32(a0)
        return TA(kind, JSArrayBuffer(n * size), 0, n)
    if t is JSArrayBuffer:
        off = to_uint32(args[1]) if len(args) > 1 and args[1] is not None else 0
        if len(args) > 2 and args[2] is not None:
            n = to_uint32(args[2])
        else:
            if (len(a0.data) - off) % size:
                raise JsRuntimeError("RangeError: buffer length is not a multiple of the element size")
            n = (len(a0.data) - off) // size
        if off % size or off + n * size > len(a0.data):
            raise JsRuntimeError("RangeError: view outside its buffer")
        return TA(kind, a0, off, n)
    if t is TA or t is JSArray:
        vals = a0.mv.tolist() if t is TA else list(a0)
        out = TA(kind, JSArrayBuffer(len(vals) * size), 0, len(vals))
        for i, v in enumerate(vals):
            out.mv[i] = out.conv(v)
        return out
    raise JsRuntimeError(f"new {kind}({t.__name__}) is outside the subset")


def _ta_method(o, name, args):
    if name == "fill":
        cv = o.conv(args[0] if args else None)
        s = _rel_index(args[1] if len(args) > 1 else 0, o.n)
        e = _rel_index(args[2] if len(args) > 2 and args[2] is not None else o.n, o.n)
        for i in range(s, e):
            o.mv[i] = cv
        return o
    if name == "set":
        src = args[0]
        off = to_uint32(args[1]) if len(args) > 1 and args[1] is not None else 0
        n = len(src)
        if off + n > o.n:
            raise JsRuntimeError("RangeError: offset is out of bounds")
        if type(src) is TA and src.fmt == o.fmt:
            data = src.mv
            if src.buffer is o.buffer:
                data = memoryview(bytearray(src.mv.tobytes())).cast(src.fmt)
            o.mv[off:off + n] = data
        else:
            vals = src.mv.tolist() if type(src) is TA else list(src)
            for i in range(n):
                o.mv[off + i] = o.conv(vals[i])
        return None
    if name in ("subarray", "slice"):
        s = _rel_index(args[0] if args else 0, o.n)
        e = _rel_index(args[1] if len(args) > 1 and args[1] is not None else o.n, o.n)
        e = max(e, s)
        if name == "subarray":
            return TA(o.kind, o.buffer, o.offset + s * o.size, e - s)
        out = TA(o.kind, JSArrayBuffer((e - s) * o.size), 0, e - s)
        out.mv[:] = o.mv[s:e]
        return out
    raise JsRuntimeError(f"typed-array method {name!r} is outside the subset")


def _array_method(o, name, args):
    if name == "push":
        o.extend(args)
        return len(o)
    if name == "pop":
        return o.pop() if o else None
    if name == "filter":
        out = JSArray()
        for i, v in enumerate(list(o)):
            if truthy(call_value(args[0], None, [v, i, o])):
                out.append(v)
        return out
    if name == "map":
        return JSArray(call_value(args[0], None, [v, i, o]) for i, v in enumerate(list(o)))
    if name == "slice":
        s = _rel_index(args[0] if args else 0, len(o))
        e = _rel_index(args[1] if len(args) > 1 and args[1] is not None else len(o), len(o))
        return JSArray(o[s:max(s, e)])
    raise JsRuntimeError(f"array method {name!r} is outside the subset")


def _buffer_method(o, name, args):
    if name == "slice":
        n = len(o.data)
        s = _rel_index(args[0] if args else 0, n)
        e = _rel_index(args[1] if len(args) > 1 and args[1] is not None else n, n)
        return JSArrayBuffer(bytearray(o.data[s:max(s, e)]))
    raise JsRuntimeError(f"ArrayBuffer method {name!r} is outside the subset")


_ARRAYBUFFER, _ARRAY, _OBJECT, _BOOLEAN = object(), object(), object(), object()


def call_value(f, this, args):
    t = type(f)
    if t is JSFunction:
        return f.fn(this, *args)
    if f is _BOOLEAN:
        return truthy(args[0] if args else None)
    if callable(f) and t is not JSClass:
        return f(*args)
    raise JsRuntimeError(f"TypeError: {to_string(f)} is not a function")


def call_method(o, name, args):
    t = type(o)
    if t is JSObject:
        f = get_prop(o, name)
        if f is None:
            raise JsRuntimeError(f"TypeError: {name} is not a function")
        return call_value(f, o, args)
    if t is TA:
        return _ta_method(o, name, args)
    if t is JSArray:
        return _array_method(o, name, args)
    if t is JSArrayBuffer:
        return _buffer_method(o, name, args)
    if t is Namespace:
        f = o.members.get(name)
        if f is None:
            raise JsRuntimeError(f"{o.name}.{name} is outside the subset")
        return call_value(f, o, args)
    if t is JSClass and name in o.statics:
        return call_value(o.statics[name], o, args)
    raise JsRuntimeError(f"TypeError: cannot call {name!r} on {to_string(o)}")


def construct(c, args):
    if type(c) is JSClass:
        obj = JSObject(proto=c)
        if c.ctor is not None:
            c.ctor(obj, *args)
        return obj
    if type(c) is str and c in _TA_KINDS:
        return _new_ta(c, args)
    if c is _ARRAYBUFFER:
        return JSArrayBuffer(to_uint32(args[0]) if args else 0)
    if c is _ARRAY:
        if len(args) == 1 and type(args[0]) in (int, float):
            return JSArray([None] * to_uint32(args[0]))
        return JSArray(args)
    if c is _OBJECT:
        return JSObject()
    raise JsRuntimeError(f"TypeError: {to_string(c)} is not a constructor")


def _math_min(*a):
    out = math.inf
    for v in a:
        v = to_number(v)
        if v != v:
            return math.nan
        if v < out or (v == 0 and out == 0 and math.copysign(1.0, v) < 0):
            out = v
    return out


def _math_max(*a):
    out = -math.inf
    for v in a:
        v = to_number(v)
        if v != v:
            return math.nan
        if v > out or (v == 0 and out == 0 and math.copysign(1.0, out) < 0):
            out = v
    return out


def _math_floor(v=None):
    v = to_number(v)
    if type(v) is int or not math.isfinite(v) or v == 0:
        return v
    return math.floor(v)


def _math_sqrt(v=None):
    v = to_number(v)
    return math.sqrt(v) if v >= 0 else math.nan


def _math_fround(v=None):
    v = float(to_number(v))
    if not math.isfinite(v):
        return v
    try:
        return struct.unpack("<f", struct.pack("<f", v))[0]
    except OverflowError:
        return math.copysign(math.inf, v)


def _is_finite(v=None):
    return type(v) is int or (type(v) is float and math.isfinite(v))


def _console(*a):
    print(" ".join(to_string(x) for x in a))


GLOBALS = {
    "Math": Namespace("Math", min=_math_min, max=_math_max, floor=_math_floor, sqrt=_math_sqrt,
                      abs=lambda v=None: abs(to_number(v)), fround=_math_fround, PI=math.pi),
    "Number": Namespace("Number", isFinite=_is_finite,
                        isInteger=lambda v=None: _is_finite(v) and float(v).is_integer()),
    "console": Namespace("console", log=_console, warn=_console, error=_console),
    "Infinity": math.inf, "NaN": math.nan, "undefined": None,
    "ArrayBuffer": _ARRAYBUFFER, "Array": _ARRAY, "Object": _OBJECT, "Boolean": _BOOLEAN,
    "isFinite": lambda v=None: math.isfinite(to_number(v)),
}
for _kind in _TA_KINDS:
    GLOBALS[_kind] = _kind


# ---------------------------------------------------------------------------- code generation

_STMT_KINDS = {"var", "funcdecl", "class", "if", "for", "forof", "while", "dowhile", "return",
               "break", "continue", "block", "expr", "empty", "export", "import"}


class _FnScope:
    """Bindings of one JS function: a stack of block scopes mapping JS names to
    Python names that are unique across the module."""

    def __init__(self, parent, is_arrow, gen):
        self.parent, self.is_arrow, self.gen = parent, is_arrow, gen
        self.blocks = [{}]
        self.pynames = set()
        self.nonlocals = set()

    def declare(self, name):
        base = "v_" + name.replace("$", "_S")
        py, k = base, 0
        while py in self.gen.pynames:
            k += 1
            py = f"{base}_{k}"
        self.gen.pynames.add(py)
        self.pynames.add(py)
        self.blocks[-1][name] = py
        return py

    def lookup(self, name):
        for b in reversed(self.blocks):
            if name in b:
                return b[name]
        return None


def _pure(e):
    """No side effects anywhere inside (no call, new, assignment or update)."""
    k = e[0]
    if k in ("num", "str", "bool", "null", "id", "this"):
        return True
    if k in ("call", "new", "assign", "update", "funcexpr"):
        return False
    if k == "member":
        return _pure(e[1])
    if k == "index":
        return _pure(e[1]) and _pure(e[2])
    if k == "unary":
        return _pure(e[2])
    if k in ("bin", "logic"):
        return _pure(e[2]) and _pure(e[3])
    if k == "cond":
        return _pure(e[1]) and _pure(e[2]) and _pure(e[3])
    if k in ("array", "seq"):
        return all(_pure(x) for x in e[1])
    if k == "object":
        return all(_pure(v) for _, v in e[1])
    return False


def _walk(x, visit):
    """Visit every tuple node below x (function bodies included)."""
    if isinstance(x, tuple) and x and isinstance(x[0], str):
        visit(x)
        for y in x[1:]:
            _walk(y, visit)
    elif isinstance(x, (list, tuple)):
        for y in x:
            _walk(y, visit)


def _assigned(stmts):
    """JS names assigned or updated anywhere in these statements."""
    out = set()

    def visit(n):
        if n[0] == "assign" and n[2][0] == "id":
            out.add(n[2][1])
        elif n[0] == "update" and n[3][0] == "id":
            out.add(n[3][1])
        elif n[0] == "forof":
            out.add(n[2])
    _walk(stmts, visit)
    return out


def _has_functions(stmts):
    found = []
    _walk(stmts, lambda n: found.append(n) if n[0] in ("funcexpr", "funcdecl", "class") else None)
    return bool(found)


def _body(s):
    return s[1] if s[0] == "block" else [s]


def _has_continue(stmts):
    """A `continue` that belongs to the loop around these statements."""
    for s in stmts:
        if s[0] == "continue":
            return True
        if s[0] == "if" and (_has_continue(_body(s[2])) or (s[3] is not None and _has_continue(_body(s[3])))):
            return True
        if s[0] == "block" and _has_continue(s[1]):
            return True
    return False


_COMPOUND = {"+=": "op_add", "-=": "op_sub", "*=": "op_mul", "/=": "op_div", "%=": "op_mod",
             "<<=": "op_shl", ">>=": "op_sar", ">>>=": "op_shr", "&=": "op_and", "|=": "op_or",
             "^=": "op_xor", "**=": "op_pow"}
_BINOPS = {"+": "op_add", "-": "op_sub", "*": "op_mul", "/": "op_div", "%": "op_mod", "**": "op_pow",
           "|": "op_or", "&": "op_and", "^": "op_xor", "<<": "op_shl", ">>": "op_sar", ">>>": "op_shr",
           "===": "strict_eq", "==": "loose_eq", "<": "op_lt", ">": "op_gt", "<=": "op_le",
           ">=": "op_ge"}


class CodeGen:
    def __init__(self):
        self.tmp = 0
        self.globals_used = set()
        self.exports = []
        self.pynames = set()   # every Python name handed out in the module
        self.loops = []        # per enclosing loop: the lines a `continue` runs first
        self.pre = [[]]        # per statement: defs of the function expressions it holds

    def fresh(self, base="t"):
        self.tmp += 1
        return f"_{base}{self.tmp}"

    def resolve(self, fs, name, write=False):
        py = fs.lookup(name)
        if py is not None:
            return py
        s = fs.parent
        while s is not None:
            py = s.lookup(name)
            if py is not None:
                if write:   # every function between the binding and here needs the cell
                    m = fs
                    while m is not s:
                        m.nonlocals.add(py)
                        m = m.parent
                return py
            s = s.parent
        if name in GLOBALS or name == "self":
            if write:
                raise JsRuntimeError(f"assigning the global {name!r} is outside the subset")
            self.globals_used.add(name)
            return "G_" + name
        raise JsSyntaxError(f"{name!r} is not declared")

    # expressions
    def expr(self, fs, e):
        k = e[0]
        if k == "num":
            v = e[1]
            if type(v) is float and v.is_integer() and abs(v) < 2 ** 53:
                return repr(int(v))
            return repr(v) if type(v) is int or math.isfinite(v) else "math.inf"
        if k == "str":
            return repr(e[1])
        if k == "bool":
            return repr(e[1])
        if k == "null":
            return "NULL"
        if k == "this":
            return "js_this"
        if k == "id":
            if e[1] == "undefined" and fs.lookup("undefined") is None:
                return "None"
            return self.resolve(fs, e[1])
        if k == "array":
            return "JSArray([" + ", ".join(self.expr(fs, x) for x in e[1]) + "])"
        if k == "object":
            return "JSObject({" + ", ".join(f"{key!r}: {self.expr(fs, v)}" for key, v in e[1]) + "})"
        if k == "member":
            return f"get_prop({self.expr(fs, e[1])}, {e[2]!r})"
        if k == "index":
            return f"get_key({self.expr(fs, e[1])}, {self.expr(fs, e[2])})"
        if k == "call":
            callee, args = e[1], ", ".join(self.expr(fs, a) for a in e[2])
            if callee[0] == "member":
                return f"call_method({self.expr(fs, callee[1])}, {callee[2]!r}, [{args}])"
            if callee[0] == "index":
                return f"call_method({self.expr(fs, callee[1])}, to_string({self.expr(fs, callee[2])}), [{args}])"
            return f"call_value({self.expr(fs, callee)}, None, [{args}])"
        if k == "new":
            return f"construct({self.expr(fs, e[1])}, [{', '.join(self.expr(fs, a) for a in e[2])}])"
        if k == "unary":
            op, a = e[1], self.expr(fs, e[2])
            if op == "!":
                return f"(not {self.cond(fs, e[2])})"
            if op == "-":
                return f"(-{a})" if e[2][0] == "num" and e[2][1] != 0 else f"op_neg({a})"
            if op == "+":
                return f"to_number({a})"
            if op == "~":
                return f"op_not({a})"
            if op == "typeof":
                return f"typeof({a})"
            return f"(({a}), None)[1]"   # void
        if k == "bin":
            op, a, b = e[1], self.expr(fs, e[2]), self.expr(fs, e[3])
            if op == "!==":
                return f"(not strict_eq({a}, {b}))"
            if op == "!=":
                return f"(not loose_eq({a}, {b}))"
            if op not in _BINOPS:
                raise JsSyntaxError(f"operator {op!r} is outside the subset")
            return f"{_BINOPS[op]}({a}, {b})"
        if k == "logic":
            t = self.fresh()
            a, b = self.expr(fs, e[2]), self.expr(fs, e[3])
            if e[1] == "&&":
                return f"({b} if truthy({t} := {a}) else {t})"
            if e[1] == "||":
                return f"({t} if truthy({t} := {a}) else {b})"
            return f"({b} if (({t} := {a}) is None or {t} is NULL) else {t})"
        if k == "cond":
            return f"({self.expr(fs, e[2])} if {self.cond(fs, e[1])} else {self.expr(fs, e[3])})"
        if k == "assign":
            return self.assign(fs, e)
        if k == "update":
            return self.update(fs, e)
        if k == "seq":
            return "(" + ", ".join(self.expr(fs, x) for x in e[1]) + ")[-1]"
        if k == "funcexpr":
            return self.function_value(fs, e[1], e[2], e[3], e[4])
        raise JsSyntaxError(f"expression {k!r} is outside the subset")

    def cond(self, fs, e):
        """A Python boolean for a JS condition."""
        if e[0] == "bin" and e[1] in ("<", ">", "<=", ">=", "===", "!==", "==", "!="):
            return self.expr(fs, e)
        if e[0] == "unary" and e[1] == "!":
            return self.expr(fs, e)
        if e[0] == "bool":
            return repr(e[1])
        return f"truthy({self.expr(fs, e)})"

    def assign(self, fs, e):
        op, target, value = e[1], e[2], e[3]
        if op not in ("=",) and op not in _COMPOUND:
            raise JsSyntaxError(f"{op} is outside the subset")
        v = self.expr(fs, value)
        if target[0] == "id":
            py = self.resolve(fs, target[1], write=True)
            return f"({py} := {v})" if op == "=" else f"({py} := {_COMPOUND[op]}({py}, {v}))"
        obj = self.expr(fs, target[1])
        if target[0] == "member":
            key, setter, aug = repr(target[2]), "set_prop", "aug_prop"
        else:
            key, setter, aug = self.expr(fs, target[2]), "set_key", "aug_key"
        if op == "=":
            return f"{setter}({obj}, {key}, {v})"
        if _pure(value):
            return f"{aug}({obj}, {key}, {_COMPOUND[op]}, {v})"
        return f"{aug}_lazy({obj}, {key}, {_COMPOUND[op]}, lambda: {v})"

    def update(self, fs, e):
        op, prefix, target = e[1], e[2], e[3]
        d = 1 if op == "++" else -1
        if target[0] == "id":
            py = self.resolve(fs, target[1], write=True)
            if prefix:
                return f"({py} := to_number({py}) + {d})"
            t = self.fresh()
            return f"(({t} := to_number({py})), ({py} := {t} + {d}))[0]"
        obj = self.expr(fs, target[1])
        if target[0] == "member":
            return f"upd_prop({obj}, {target[2]!r}, {d}, {prefix})"
        return f"upd_key({obj}, {self.expr(fs, target[2])}, {d}, {prefix})"

    def expr_stmt(self, fs, e):
        if e[0] == "assign" and e[2][0] == "id" and e[1] == "=":
            return f"{self.resolve(fs, e[2][1], write=True)} = {self.expr(fs, e[3])}"
        if e[0] == "update" and e[3][0] == "id":
            py = self.resolve(fs, e[3][1], write=True)
            return f"{py} = to_number({py}) + {1 if e[1] == '++' else -1}"
        return self.expr(fs, e)

    # statements
    def stmts(self, fs, body, out, ind):
        # a block's bindings exist before its first statement runs (hoisting)
        for s in body:
            d = s[1] if s[0] == "export" else s
            names = []
            if d[0] in ("funcdecl", "class"):
                names = [d[1]]
            elif d[0] == "var":
                names = [n for n, _ in d[2]]
            elif d[0] == "import":
                names = [local for _, local in d[1]]
            for n in names:
                if fs.blocks[-1].get(n) is None:
                    fs.declare(n)
        funcs = [s for s in body if (s[1] if s[0] == "export" else s)[0] == "funcdecl"]
        for s in funcs + [s for s in body if s not in funcs]:
            self.stmt(fs, s, out, ind)

    def block(self, fs, body, out, ind):
        fs.blocks.append({})
        n0 = len(out)
        self.stmts(fs, body, out, ind)
        if len(out) == n0:
            out.append(ind + "pass")
        fs.blocks.pop()

    def loop_body(self, fs, body, out, ind, cont_lines):
        self.loops.append(cont_lines)
        self.block(fs, body, out, ind)
        self.loops.pop()

    def stmt(self, fs, s, out, ind):
        """One statement; the defs of function expressions inside it come first."""
        self.pre.append([])
        lines = []
        self._stmt(fs, s, lines, ind)
        for d in self.pre.pop():
            out.extend(ind + line for line in d)
        out.extend(lines)

    def _stmt(self, fs, s, out, ind):
        k = s[0]
        if k == "export":
            d = s[1]
            if d[0] in ("funcdecl", "class"):
                self.exports.append(d[1])
            elif d[0] == "var":
                self.exports.extend(n for n, _ in d[2])
            else:
                raise JsSyntaxError("this export form is outside the subset")
            self._stmt(fs, d, out, ind)
        elif k == "import":
            for imported, local in s[1]:
                py = fs.blocks[-1].get(local) or fs.declare(local)
                out.append(f"{ind}{py} = IMPORTS[{s[2]!r}][{imported!r}]")
        elif k == "var":
            for name, init in s[2]:
                v = "None" if init is None else self.expr(fs, init)
                py = fs.blocks[-1].get(name) or (fs.lookup(name) if s[1] == "var" else None) or fs.declare(name)
                out.append(f"{ind}{py} = {v}")
        elif k == "funcdecl":
            py = fs.blocks[-1].get(s[1]) or fs.declare(s[1])
            fname = self.fresh("f")
            self.function_def(fs, fname, s[2], s[3], False, out, ind)
            out.append(f"{ind}{py} = JSFunction({fname}, {s[1]!r})")
        elif k == "class":
            py = fs.blocks[-1].get(s[1]) or fs.declare(s[1])
            ctor, parts = "None", {"method": {}, "get": {}, "set": {}, "static": {}}
            for kind, name, params, body in s[2]:
                fname = self.fresh("m")
                self.function_def(fs, fname, params, body, False, out, ind)
                if kind == "ctor":
                    ctor = fname
                elif kind in ("method", "static"):
                    parts[kind][name] = f"JSFunction({fname}, {name!r})"
                else:
                    parts[kind][name] = fname

            def d(m):
                return "{" + ", ".join(f"{a!r}: {b}" for a, b in m.items()) + "}"
            out.append(f"{ind}{py} = JSClass({s[1]!r}, {ctor}, {d(parts['method'])}, {d(parts['get'])}, "
                       f"{d(parts['set'])}, {d(parts['static'])})")
        elif k == "expr":
            out.append(ind + self.expr_stmt(fs, s[1]))
        elif k == "empty":
            pass
        elif k == "block":
            self.block(fs, s[1], out, ind)
        elif k == "if":
            out.append(f"{ind}if {self.cond(fs, s[1])}:")
            self.block(fs, _body(s[2]), out, ind + "    ")
            alt = s[3]
            while alt is not None and alt[0] == "if":
                out.append(f"{ind}elif {self.cond(fs, alt[1])}:")
                self.block(fs, _body(alt[2]), out, ind + "    ")
                alt = alt[3]
            if alt is not None:
                out.append(f"{ind}else:")
                self.block(fs, _body(alt), out, ind + "    ")
        elif k == "while":
            out.append(f"{ind}while {self.cond(fs, s[1])}:")
            self.loop_body(fs, _body(s[2]), out, ind + "    ", [])
        elif k == "dowhile":
            if _has_continue(_body(s[1])):
                raise JsSyntaxError("continue inside do-while is outside the subset")
            out.append(f"{ind}while True:")
            self.loop_body(fs, _body(s[1]), out, ind + "    ", [])
            out.append(f"{ind}    if not {self.cond(fs, s[2])}:")
            out.append(f"{ind}        break")
        elif k == "for":
            self.for_loop(fs, s, out, ind)
        elif k == "forof":
            fs.blocks.append({})
            it = self.expr(fs, s[3])
            py = fs.declare(s[2])
            out.append(f"{ind}for {py} in iterate({it}):")
            self.loop_body(fs, _body(s[4]), out, ind + "    ", [])
            fs.blocks.pop()
        elif k == "return":
            out.append(f"{ind}return {'None' if s[1] is None else self.expr(fs, s[1])}")
        elif k == "break":
            out.append(ind + "break")
        elif k == "continue":
            out.extend(ind + line for line in (self.loops[-1] if self.loops else []))
            out.append(ind + "continue")
        else:
            raise JsSyntaxError(f"statement {k!r} is outside the subset")

    def for_loop(self, fs, s, out, ind):
        init, test, update, body = s[1], s[2], s[3], _body(s[4])
        fs.blocks.append({})
        fast = self.counted(init, test, update, body)
        if fast is not None:
            var, start, bound, inclusive = fast
            stop = f"range_stop({self.expr(fs, bound)}, {inclusive})"
            py = fs.declare(var)
            out.append(f"{ind}for {py} in range({start}, {stop}):")
            self.loop_body(fs, body, out, ind + "    ", [])
        else:
            if init is not None:
                if init[0] == "var":
                    self._stmt(fs, init, out, ind)
                else:
                    out.append(ind + self.expr_stmt(fs, init[1]))
            upd = [] if update is None else [self.expr_stmt(fs, update)]
            out.append(f"{ind}while {'True' if test is None else self.cond(fs, test)}:")
            self.loop_body(fs, body, out, ind + "    ", upd)
            out.extend(ind + "    " + line for line in upd)
        fs.blocks.pop()

    @staticmethod
    def counted(init, test, update, body):
        """`for (let i = <int>; i < b; i++)` whose body assigns neither i nor the
        bound b (a name or a literal) and declares no function: a Python range."""
        if init is None or init[0] != "var" or init[1] not in ("let", "const") or len(init[2]) != 1:
            return None
        var, start = init[2][0]
        if start is None or start[0] != "num" or type(start[1]) is not int:
            return None
        if test is None or test[0] != "bin" or test[1] not in ("<", "<=") or test[2] != ("id", var):
            return None
        if update is None or update[0] != "update" or update[1] != "++" or update[3] != ("id", var):
            return None
        assigned = _assigned(body)
        if var in assigned or _has_functions(body):
            return None
        bound = test[3]
        if not (bound[0] == "num" or (bound[0] == "id" and bound[1] not in assigned)):
            return None
        return var, start[1], bound, test[1] == "<="

    def function_def(self, fs, pyname, params, body, is_arrow, out, ind):
        inner = _FnScope(fs, is_arrow, self)
        args, defaults = [], []
        for name, default in params:
            py = inner.declare(name)
            args.append(f"{py}=None")
            if default is not None:
                defaults.append((py, default))
        lines = []
        bi = ind + "    "
        for py, default in defaults:
            lines.append(f"{bi}if {py} is None:")
            lines.append(f"{bi}    {py} = {self.expr(inner, default)}")
        saved = self.loops
        self.loops = []
        self.stmts(inner, body, lines, bi)
        self.loops = saved
        # an arrow function keeps the `this` of the function around it (a closure)
        this_arg = "_arrow_this" if is_arrow else "js_this"
        out.append(f"{ind}def {pyname}({', '.join([this_arg] + args + ['*_extra'])}):")
        nl = sorted(inner.nonlocals)
        if nl:
            out.append(f"{bi}nonlocal {', '.join(nl)}")
        out.extend(lines or [bi + "pass"])

    def function_value(self, fs, name, params, body, is_arrow):
        fname = self.fresh("f")
        lines = []
        self.pre.append([])
        self.function_def(fs, fname, params, body, is_arrow, lines, "")
        self.pre[-2].extend(self.pre.pop())
        self.pre[-1].append(lines)
        return f"JSFunction({fname}, {name or ''!r})"


# ---------------------------------------------------------------------------- modules


def compile_module(src):
    """Python source of `MODULE(IMPORTS, G_self) -> exports` for an ES module."""
    ast = Parser(src).program()
    gen = CodeGen()
    top = _FnScope(None, False, gen)
    body = []
    gen.stmts(top, ast, body, "    ")
    lines = ["def MODULE(IMPORTS, G_self):", "    js_this = None"]
    lines += [f"    G_{g} = GLOBALS[{g!r}]" for g in sorted(gen.globals_used) if g != "self"]
    lines += body
    lines.append("    return {" + ", ".join(f"{n!r}: {top.lookup(n)}" for n in gen.exports) + "}")
    return "\n".join(lines) + "\n"


def _run(src, name, imports, self_object):
    ns = {k: v for k, v in globals().items() if not k.startswith("__")}
    exec(compile(compile_module(src), f"<js:{name}>", "exec"), ns)
    return ns["MODULE"](imports, JSObject() if self_object is None else self_object)


def run_source(src, imports=None, self_object=None):
    """Run module source text; returns its exports."""
    return _run(src, "source", imports or {}, self_object)


def load_module(path, self_object=None, _cache=None):
    """Run an ES module file; returns its exports (dict). Relative imports are
    loaded from the module's directory. ``self_object`` is the worker global
    ``self`` (a JSObject) for modules that use it."""
    cache = {} if _cache is None else _cache
    path = os.path.abspath(path)
    if path not in cache:
        src = open(path, encoding="utf-8").read()
        imports = {}
        for spec in re.findall(r"""^\s*import\s*\{[^}]*\}\s*from\s*['"]([^'"]+)['"]""", src, re.M):
            imports[spec] = load_module(os.path.join(os.path.dirname(path), spec), self_object, cache)
        cache[path] = _run(src, os.path.basename(path), imports, self_object)
    return cache[path]


# ---------------------------------------------------------------------------- numpy bridges

_NP = {"f": "<f4", "d": "<f8", "i": "<i4", "I": "<u4", "B": "u1", "b": "i1", "h": "<i2", "H": "<u2"}
_KIND_OF_NP = {"float32": "Float32Array", "float64": "Float64Array", "int32": "Int32Array",
               "uint32": "Uint32Array", "uint8": "Uint8Array", "int8": "Int8Array",
               "int16": "Int16Array", "uint16": "Uint16Array"}


def from_numpy(a):
    """A typed array holding a copy of a numpy array (in its own ArrayBuffer)."""
    import numpy as np

    a = np.ascontiguousarray(a)
    return TA(_KIND_OF_NP[str(a.dtype)], JSArrayBuffer(bytearray(a.reshape(-1).tobytes())), 0, a.size)


def to_numpy(v):
    """A numpy copy of a typed array or a (nested) JS array of numbers."""
    import numpy as np

    if type(v) is TA:
        return np.frombuffer(bytes(v.buffer.data[v.offset:v.offset + v.n * v.size]), _NP[v.fmt]).copy()
    if type(v) is JSArray:
        return np.array([to_numpy(x) if type(x) in (JSArray, TA) else x for x in v])
    raise TypeError(type(v))
