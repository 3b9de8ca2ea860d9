"""A small JavaScript-subset engine for running the reference's solver sources.

TEST INFRASTRUCTURE. No JavaScript engine exists on this machine, so the
golden vectors in tests/golden are produced by running the unmodified
reference files (js/lbm.js, js/shapes.js, js/voxel.js) through this module:
it parses the subset of ECMAScript those files use and translates it to
Python source, which is then executed. Numbers follow JS semantics where the
files depend on them: arithmetic is IEEE double (Python float; integer
literals stay exact Python ints, which agree with doubles below 2**53),
typed-array stores round through the element type (`array.array`), `| 0`
and the other bitwise operators go through ToInt32, and `%` keeps the sign
of the dividend.

Known differences from a real engine, none of which the solver files rely
on: truthiness of empty arrays / objects and of NaN follows Python; `null`
and `undefined` are both None; Math.sin / cos / pow come from the host libm
(V8 uses fdlibm, which can differ in the last bit), so fixtures record the
rotation matrices they were given rather than recomputing them.
"""
from __future__ import annotations

import array
import functools
import keyword
import math
import re

# ============================================================================ tokenizer
_PUNCT = sorted("""
>>>= ... === !== **= <<= >>= >>> => == != <= >= && || ?? ?. ++ -- += -= *= /= %= &= |= ^= << >> **
{ } ( ) [ ] ; , < > + - * / % & | ^ ! ~ ? : = .
""".split(), key=len, reverse=True)

_TOKEN_RE = re.compile(r"""
  (?P<ws>[ \t\r\n]+)
| (?P<lc>//[^\n]*)
| (?P<bc>/\*.*?\*/)
| (?P<num>0[xX][0-9a-fA-F]+|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)
| (?P<str>'(?:[^'\\\n]|\\.)*'|"(?:[^"\\\n]|\\.)*")
| (?P<tpl>`(?:[^`\\]|\\.)*`)
| (?P<id>[A-Za-z_$][\w$]*)
| (?P<p>""" + "|".join(re.escape(p) for p in _PUNCT) + r""")
""", re.S | re.X)

KEYWORDS = {"var", "let", "const", "function", "return", "if", "else", "for", "while", "do",
            "break", "continue", "new", "class", "extends", "this", "typeof", "instanceof",
            "in", "of", "switch", "case", "default", "throw", "try", "catch", "finally", "null",
            "true", "false", "void", "delete", "static", "get", "set", "super"}


class Tok:
    __slots__ = ("kind", "val", "pos", "nl")

    def __init__(self, kind, val, pos, nl):
        self.kind, self.val, self.pos, self.nl = kind, val, pos, nl

    def __repr__(self):
        return f"Tok({self.kind},{self.val!r})"


def tokenize(src: str) -> list[Tok]:
    out, pos, nl = [], 0, False
    while pos < len(src):
        m = _TOKEN_RE.match(src, pos)
        if not m:
            raise SyntaxError(f"bad character at {pos}: {src[pos:pos + 20]!r}")
        kind = m.lastgroup
        text = m.group(kind)
        if kind in ("ws", "lc", "bc"):
            if "\n" in text:
                nl = True
        else:
            if kind == "id" and text in KEYWORDS:
                kind = "kw"
            out.append(Tok(kind, text, pos, nl))
            nl = False
        pos = m.end()
    out.append(Tok("eof", None, pos, True))
    return out


# ============================================================================ parser (AST as tuples)
class Parser:
    def __init__(self, src: str):
        self.t = tokenize(src)
        self.i = 0

    # -- token helpers
    def peek(self, k=0):
        return self.t[min(self.i + k, len(self.t) - 1)]

    def at(self, val, k=0):
        tk = self.peek(k)
        return tk.kind in ("p", "kw") and tk.val == val

    def eat(self, val):
        if self.at(val):
            self.i += 1
            return True
        return False

    def expect(self, val):
        if not self.eat(val):
            tk = self.peek()
            raise SyntaxError(f"expected {val!r} at {tk.pos}, got {tk.val!r}")

    def ident(self):
        tk = self.peek()
        if tk.kind == "id" or (tk.kind == "kw" and tk.val in ("of", "get", "set", "static")):
            self.i += 1
            return tk.val
        raise SyntaxError(f"expected identifier at {tk.pos}, got {tk.val!r}")

    def semi(self):
        self.eat(";")

    # -- program
    def program(self):
        body = []
        while self.peek().kind != "eof":
            body.append(self.statement())
        return ("Program", body)

    def block(self):
        self.expect("{")
        body = []
        while not self.at("}"):
            body.append(self.statement())
        self.expect("}")
        return ("Block", body)

    def statement(self):
        tk = self.peek()
        if tk.kind == "p" and tk.val == "{":
            return self.block()
        if tk.kind == "p" and tk.val == ";":
            self.i += 1
            return ("Empty",)
        if tk.kind == "kw":
            v = tk.val
            if v in ("var", "let", "const"):
                d = self.var_decl()
                self.semi()
                return d
            if v == "function":
                self.i += 1
                name = self.ident()
                params, body = self.func_rest()
                return ("FuncDecl", name, params, body)
            if v == "class":
                return self.class_decl()
            if v == "return":
                self.i += 1
                arg = None
                if not (self.at(";") or self.at("}") or self.peek().nl):
                    arg = self.expression()
                self.semi()
                return ("Return", arg)
            if v == "if":
                self.i += 1
                self.expect("(")
                test = self.expression()
                self.expect(")")
                cons = self.statement()
                alt = self.statement() if self.eat("else") else None
                return ("If", test, cons, alt)
            if v == "for":
                return self.for_stmt()
            if v == "while":
                self.i += 1
                self.expect("(")
                test = self.expression()
                self.expect(")")
                return ("While", test, self.statement())
            if v == "do":
                self.i += 1
                body = self.statement()
                self.expect("while")
                self.expect("(")
                test = self.expression()
                self.expect(")")
                self.semi()
                return ("DoWhile", body, test)
            if v == "break":
                self.i += 1
                self.semi()
                return ("Break",)
            if v == "continue":
                self.i += 1
                self.semi()
                return ("Continue",)
            if v == "throw":
                self.i += 1
                arg = self.expression()
                self.semi()
                return ("Throw", arg)
            if v == "switch":
                return self.switch_stmt()
            if v == "try":
                self.i += 1
                blk = self.block()
                param = handler = fin = None
                if self.eat("catch"):
                    if self.eat("("):
                        param = self.ident()
                        self.expect(")")
                    handler = self.block()
                if self.eat("finally"):
                    fin = self.block()
                return ("Try", blk, param, handler, fin)
        e = self.expression()
        self.semi()
        return ("Expr", e)

    def var_decl(self):
        kind = self.peek().val
        self.i += 1
        decls = []
        while True:
            if self.at("{") or self.at("["):
                target = self.pattern()
            else:
                target = ("Id", self.ident())
            init = self.assign() if self.eat("=") else None
            decls.append((target, init))
            if not self.eat(","):
                break
        return ("Var", kind, decls)

    def pattern(self):
        if self.eat("{"):
            names = []
            while not self.at("}"):
                key = self.ident()
                local = self.ident() if self.eat(":") else key
                names.append((key, local))
                if not self.eat(","):
                    break
            self.expect("}")
            return ("ObjPat", names)
        self.expect("[")
        names = []
        while not self.at("]"):
            names.append(None if self.at(",") else self.ident())
            if not self.eat(","):
                break
        self.expect("]")
        return ("ArrPat", names)

    def for_stmt(self):
        self.expect("for")
        self.expect("(")
        init = None
        if self.at("var") or self.at("let") or self.at("const"):
            if (self.peek(1).kind == "id" and self.peek(2).kind == "kw"
                    and self.peek(2).val in ("of", "in")):
                self.i += 1
                name = self.ident()
                kind = self.peek().val
                self.i += 1
                it = self.expression()
                self.expect(")")
                return ("ForOf" if kind == "of" else "ForIn", name, it, self.statement())
            init = self.var_decl()
        elif not self.at(";"):
            init = ("Expr", self.expression())
        self.expect(";")
        test = None if self.at(";") else self.expression()
        self.expect(";")
        update = None if self.at(")") else self.expression()
        self.expect(")")
        return ("For", init, test, update, self.statement())

    def switch_stmt(self):
        self.expect("switch")
        self.expect("(")
        disc = self.expression()
        self.expect(")")
        self.expect("{")
        cases = []
        while not self.at("}"):
            if self.eat("default"):
                test = None
            else:
                self.expect("case")
                test = self.expression()
            self.expect(":")
            body = []
            while not (self.at("case") or self.at("default") or self.at("}")):
                body.append(self.statement())
            cases.append((test, body))
        self.expect("}")
        return ("Switch", disc, cases)

    def class_decl(self):
        self.expect("class")
        name = self.ident()
        base = None
        if self.eat("extends"):
            base = self.lhs()
        self.expect("{")
        members = []
        while not self.at("}"):
            if self.eat(";"):
                continue
            static = False
            if self.at("static") and not self.at("(", 1):
                self.i += 1
                static = True
            kind = "method"
            if (self.at("get") or self.at("set")) and not self.at("(", 1):
                kind = self.peek().val
                self.i += 1
            mname = self.ident()
            params, body = self.func_rest()
            members.append((kind, static, mname, params, body))
        self.expect("}")
        return ("Class", name, base, members)

    def func_rest(self):
        self.expect("(")
        params = []
        while not self.at(")"):
            if self.at("..."):
                self.i += 1
                params.append(("rest", self.ident()))
            else:
                pname = self.ident()
                default = self.assign() if self.eat("=") else None
                params.append(("p", pname, default))
            if not self.eat(","):
                break
        self.expect(")")
        return params, self.block()

    # -- expressions
    def expression(self):
        e = self.assign()
        if self.at(","):
            seq = [e]
            while self.eat(","):
                seq.append(self.assign())
            return ("Seq", seq)
        return e

    def arrow_ahead(self):
        """True when the tokens at the cursor start an arrow function."""
        tk = self.peek()
        if tk.kind == "id" and self.at("=>", 1):
            return True
        if not self.at("("):
            return False
        depth, j = 0, self.i
        while j < len(self.t):
            v = self.t[j]
            if v.kind == "p" and v.val in "([{":
                depth += 1
            elif v.kind == "p" and v.val in ")]}":
                depth -= 1
                if depth == 0:
                    nxt = self.t[j + 1]
                    return nxt.kind == "p" and nxt.val == "=>"
            j += 1
        return False

    def arrow(self):
        if self.peek().kind == "id":
            params = [("p", self.ident(), None)]
        else:
            self.expect("(")
            params = []
            while not self.at(")"):
                pname = self.ident()
                default = self.assign() if self.eat("=") else None
                params.append(("p", pname, default))
                if not self.eat(","):
                    break
            self.expect(")")
        self.expect("=>")
        if self.at("{"):
            return ("Arrow", params, self.block(), False)
        return ("Arrow", params, self.assign(), True)

    ASSIGN_OPS = {"=", "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "<<=", ">>=", ">>>=", "**="}

    def assign(self):
        if self.arrow_ahead():
            return self.arrow()
        left = self.conditional()
        tk = self.peek()
        if tk.kind == "p" and tk.val in self.ASSIGN_OPS:
            self.i += 1
            right = self.assign()
            return ("Assign", tk.val, left, right)
        return left

    def conditional(self):
        test = self.binary(0)
        if self.eat("?"):
            cons = self.assign()
            self.expect(":")
            alt = self.assign()
            return ("Cond", test, cons, alt)
        return test

    BIN_PREC = [
        {"??"}, {"||"}, {"&&"}, {"|"}, {"^"}, {"&"}, {"==", "!=", "===", "!=="},
        {"<", ">", "<=", ">=", "instanceof", "in"}, {"<<", ">>", ">>>"}, {"+", "-"},
        {"*", "/", "%"}, {"**"},
    ]

    def binary(self, level):
        if level == len(self.BIN_PREC):
            return self.unary()
        left = self.binary(level + 1)
        ops = self.BIN_PREC[level]
        while True:
            tk = self.peek()
            if tk.kind in ("p", "kw") and tk.val in ops:
                self.i += 1
                right = self.binary(level + 1)
                kind = "Logical" if tk.val in ("||", "&&", "??") else "Bin"
                left = (kind, tk.val, left, right)
            else:
                return left

    def unary(self):
        tk = self.peek()
        if tk.kind == "p" and tk.val in ("!", "-", "+", "~"):
            self.i += 1
            return ("Unary", tk.val, self.unary())
        if tk.kind == "p" and tk.val in ("++", "--"):
            self.i += 1
            return ("Update", tk.val, True, self.unary())
        if tk.kind == "kw" and tk.val in ("typeof", "void", "delete"):
            self.i += 1
            return ("Unary", tk.val, self.unary())
        e = self.postfix()
        return e

    def postfix(self):
        e = self.lhs()
        tk = self.peek()
        if tk.kind == "p" and tk.val in ("++", "--") and not tk.nl:
            self.i += 1
            return ("Update", tk.val, False, e)
        return e

    def lhs(self):
        if self.at("new"):
            self.i += 1
            callee = self.member_only()
            args = self.args() if self.at("(") else []
            e = ("New", callee, args)
        else:
            e = self.primary()
        return self.call_tail(e)

    def member_only(self):
        e = self.primary()
        while True:
            if self.eat("."):
                e = ("Member", e, self.prop_name())
            elif self.at("["):
                self.i += 1
                k = self.expression()
                self.expect("]")
                e = ("Index", e, k)
            else:
                return e

    def call_tail(self, e):
        while True:
            if self.eat("."):
                e = ("Member", e, self.prop_name())
            elif self.at("?."):
                self.i += 1
                e = ("OptMember", e, self.prop_name())
            elif self.at("["):
                self.i += 1
                k = self.expression()
                self.expect("]")
                e = ("Index", e, k)
            elif self.at("("):
                e = ("Call", e, self.args())
            else:
                return e

    def prop_name(self):
        tk = self.peek()
        if tk.kind in ("id", "kw"):
            self.i += 1
            return tk.val
        raise SyntaxError(f"bad property name at {tk.pos}")

    def args(self):
        self.expect("(")
        out = []
        while not self.at(")"):
            if self.eat("..."):
                out.append(("Spread", self.assign()))
            else:
                out.append(self.assign())
            if not self.eat(","):
                break
        self.expect(")")
        return out

    def primary(self):
        tk = self.peek()
        self.i += 1
        if tk.kind == "num":
            v = tk.val
            if v[:2] in ("0x", "0X"):
                return ("Num", int(v, 16))
            if re.fullmatch(r"\d+", v):
                return ("Num", int(v))
            return ("Num", float(v))
        if tk.kind == "str":
            return ("Str", _unescape(tk.val[1:-1]))
        if tk.kind == "tpl":
            if "${" in tk.val:
                raise SyntaxError("template substitutions are not supported")
            return ("Str", _unescape(tk.val[1:-1]))
        if tk.kind == "id":
            return ("Id", tk.val)
        if tk.kind == "kw":
            v = tk.val
            if v == "this":
                return ("This",)
            if v in ("true", "false"):
                return ("Bool", v == "true")
            if v == "null":
                return ("Null",)
            if v == "function":
                name = self.ident() if self.peek().kind == "id" else None
                params, body = self.func_rest()
                return ("FuncExpr", name, params, body)
            if v in ("of", "get", "set", "static"):
                return ("Id", v)
        if tk.kind == "p":
            if tk.val == "(":
                e = self.expression()
                self.expect(")")
                return ("Paren", e)
            if tk.val == "[":
                items = []
                while not self.at("]"):
                    if self.eat("..."):
                        items.append(("Spread", self.assign()))
                    else:
                        items.append(self.assign())
                    if not self.eat(","):
                        break
                self.expect("]")
                return ("Array", items)
            if tk.val == "{":
                return self.object_lit()
        raise SyntaxError(f"unexpected token {tk.val!r} at {tk.pos}")

    def object_lit(self):
        props = []
        while not self.at("}"):
            if self.eat("..."):
                props.append(("spread", self.assign()))
            else:
                tk = self.peek()
                if tk.kind == "p" and tk.val == "[":
                    self.i += 1
                    key = ("computed", self.assign())
                    self.expect("]")
                elif tk.kind == "str":
                    self.i += 1
                    key = _unescape(tk.val[1:-1])
                elif tk.kind == "num":
                    self.i += 1
                    key = tk.val
                else:
                    key = self.prop_name()
                if self.at("("):
                    params, body = self.func_rest()
                    props.append(("kv", key, ("FuncExpr", None, params, body)))
                elif self.eat(":"):
                    props.append(("kv", key, self.assign()))
                else:
                    props.append(("kv", key, ("Id", key)))
            if not self.eat(","):
                break
        self.expect("}")
        return ("Object", props)


def _unescape(s: str) -> str:
    return re.sub(r"\\(.)", lambda m: {"n": "\n", "t": "\t", "r": "\r"}.get(m.group(1),
                                                                       m.group(1)), s)


# ============================================================================ runtime
class JSError(Exception):
    pass


def js_error(msg=None, *_):
    return JSError(msg)


def toint32(v) -> int:
    if isinstance(v, int) and -2147483648 <= v <= 2147483647:
        return v
    if v is None or isinstance(v, str):
        v = js_tonumber(v)
    v = float(v) if not isinstance(v, int) else v
    if isinstance(v, float):
        if v != v or v in (math.inf, -math.inf):
            return 0
        v = int(v)   # truncation toward zero
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v >= (1 << 31) else v


def touint32(v) -> int:
    return toint32(v) & 0xFFFFFFFF


def js_tonumber(v):
    if v is None:
        return math.nan
    if isinstance(v, bool):
        return 1 if v else 0
    if isinstance(v, (int, float)):
        return v
    if isinstance(v, str):
        try:
            return float(v) if v.strip() else 0
        except ValueError:
            return math.nan
    return math.nan


def js_mod(a, b):
    if isinstance(a, int) and isinstance(b, int) and b != 0:
        r = abs(a) % abs(b)
        return -r if a < 0 else r
    return math.fmod(a, b) if b != 0 else math.nan


def js_div(a, b):
    try:
        return a / b
    except ZeroDivisionError:
        if a != a or a == 0:
            return math.nan
        neg = (a < 0) != (math.copysign(1.0, b) < 0)
        return -math.inf if neg else math.inf


def js_typeof(v):
    if v is None:
        return "undefined"
    if isinstance(v, bool):
        return "boolean"
    if isinstance(v, (int, float)):
        return "number"
    if isinstance(v, str):
        return "string"
    if callable(v):
        return "function"
    return "object"


class JSObject(dict):
    """A plain JS object: attribute and item access share one key space."""

    def __getattr__(self, k):
        if k.startswith("__"):
            raise AttributeError(k)
        return self.get(_unmangle(k))

    def __setattr__(self, k, v):
        self[_unmangle(k)] = v

    def __getitem__(self, k):
        return self.get(k if isinstance(k, str) else str(k))

    def __setitem__(self, k, v):
        dict.__setitem__(self, k if isinstance(k, str) else str(k), v)

    def __bool__(self):
        return True

    def __hash__(self):
        return id(self)

    def __eq__(self, other):
        return self is other


class JSArray(list):
    """A JS Array: list plus the methods the reference files call."""

    @property
    def length(self):
        return len(self)

    @length.setter
    def length(self, n):
        del self[int(n):]

    def __getitem__(self, k):
        if isinstance(k, float) and k.is_integer():
            k = int(k)
        if isinstance(k, int):
            return list.__getitem__(self, k) if 0 <= k < len(self) else None
        return list.__getitem__(self, k)

    def __setitem__(self, k, v):
        if isinstance(k, float) and k.is_integer():
            k = int(k)
        if isinstance(k, int) and k >= len(self):
            self.extend([None] * (k - len(self) + 1))
        list.__setitem__(self, k, v)

    def __bool__(self):
        return True

    def __hash__(self):
        return id(self)

    def __eq__(self, other):
        return self is other

    def push(self, *xs):
        self.extend(xs)
        return len(self)

    def sort(self, cmp=None):
        if cmp is None:
            list.sort(self, key=lambda v: str(v))
        else:
            list.sort(self, key=functools.cmp_to_key(lambda a, b: _sign(cmp(a, b))))
        return self

    def indexOf(self, v, *_):
        for i, x in enumerate(self):
            if x == v:
                return i
        return -1

    def includes(self, v, *_):
        return self.indexOf(v) >= 0

    def find(self, fn, *_):
        for i, x in enumerate(self):
            if fn(x, i, self):
                return x
        return None

    def some(self, fn, *_):
        return any(fn(x, i, self) for i, x in enumerate(self))

    def every(self, fn, *_):
        return all(fn(x, i, self) for i, x in enumerate(self))

    def map(self, fn, *_):
        return JSArray(fn(x, i, self) for i, x in enumerate(self))

    def filter(self, fn, *_):
        return JSArray(x for i, x in enumerate(self) if fn(x, i, self))

    def forEach(self, fn, *_):
        for i, x in enumerate(self):
            fn(x, i, self)

    def reduce(self, fn, *init):
        it = iter(enumerate(self))
        acc = init[0] if init else next(it)[1]
        for i, x in it:
            acc = fn(acc, x, i, self)
        return acc

    def slice(self, a=0, b=None, *_):
        return JSArray(list.__getitem__(self, slice(a, b)))

    def concat(self, *others):
        out = JSArray(self)
        for o in others:
            out.extend(o) if isinstance(o, list) else out.append(o)
        return out

    def join(self, sep=","):
        return sep.join("" if x is None else str(x) for x in self)

    def fill(self, v, a=0, b=None, *_):
        b = len(self) if b is None else b
        for i in range(a, b):
            self[i] = v
        return self


def _sign(v):
    v = js_tonumber(v)
    return 0 if v == 0 or v != v else (1 if v > 0 else -1)


def _make_typed(name, code):
    def convert(v):
        if code in "fd":
            return float(v) if not isinstance(v, float) else v
        v = toint32(v)
        bits = {"b": 8, "B": 8, "h": 16, "H": 16, "i": 32, "I": 32}[code]
        v &= (1 << bits) - 1
        if code in "bhi" and v >= 1 << (bits - 1):
            v -= 1 << bits
        return v

    class Typed(array.array):
        def __new__(cls, arg=0, *_):
            if isinstance(arg, (int, float)):
                n = int(arg)
                return array.array.__new__(cls, code, bytes(n * array.array(code).itemsize))
            return array.array.__new__(cls, code, [convert(x) for x in arg])

        @property
        def length(self):
            return len(self)

        def __bool__(self):
            return True

        def __hash__(self):
            return id(self)

        def fill(self, v, a=0, b=None, *_):
            b = len(self) if b is None else b
            cv = convert(v)
            for i in range(a, b):
                self[i] = cv
            return self

        def subarray(self, a=0, b=None, *_):
            return type(self)(list(self[a:b]))

        def slice(self, a=0, b=None, *_):
            return type(self)(list(self[a:b]))

        def sort(self, cmp=None):
            vals = sorted(self) if cmp is None else sorted(
                self, key=functools.cmp_to_key(lambda a, b: _sign(cmp(a, b))))
            self[:] = array.array(code, vals)
            return self

        def set(self, src, off=0, *_):
            for k, v in enumerate(src):
                self[off + k] = convert(v)

    Typed.__name__ = name
    return Typed


Float32Array = _make_typed("Float32Array", "f")
Float64Array = _make_typed("Float64Array", "d")
Int32Array = _make_typed("Int32Array", "i")
Uint32Array = _make_typed("Uint32Array", "I")
Int16Array = _make_typed("Int16Array", "h")
Uint16Array = _make_typed("Uint16Array", "H")
Int8Array = _make_typed("Int8Array", "b")
Uint8Array = _make_typed("Uint8Array", "B")


class _Math:
    PI = math.pi
    SQRT2 = math.sqrt(2.0)
    E = math.e
    LN2 = math.log(2.0)

    @staticmethod
    def _nums(args):
        return [js_tonumber(a) for a in args]

    def max(self, *a):
        a = self._nums(a)
        if any(x != x for x in a):
            return math.nan
        return max(a) if a else -math.inf

    def min(self, *a):
        a = self._nums(a)
        if any(x != x for x in a):
            return math.nan
        return min(a) if a else math.inf

    @staticmethod
    def floor(x, *_):
        x = js_tonumber(x)
        return math.floor(x) if isinstance(x, int) or math.isfinite(x) else x

    @staticmethod
    def ceil(x, *_):
        x = js_tonumber(x)
        return math.ceil(x) if isinstance(x, int) or math.isfinite(x) else x

    @staticmethod
    def trunc(x, *_):
        x = js_tonumber(x)
        return math.trunc(x) if isinstance(x, int) or math.isfinite(x) else x

    @staticmethod
    def round(x, *_):
        x = js_tonumber(x)
        return math.floor(x + 0.5) if math.isfinite(x) else x

    @staticmethod
    def abs(x, *_):
        return abs(js_tonumber(x))

    @staticmethod
    def sqrt(x, *_):
        x = js_tonumber(x)
        return math.sqrt(x) if x >= 0 else (math.nan if x == x and x < 0 else x)

    @staticmethod
    def sign(x, *_):
        return _sign(x)

    @staticmethod
    def hypot(*a):
        return math.hypot(*[js_tonumber(x) for x in a])

    sin = staticmethod(lambda x, *_: math.sin(x))
    cos = staticmethod(lambda x, *_: math.cos(x))
    tan = staticmethod(lambda x, *_: math.tan(x))
    atan2 = staticmethod(lambda y, x, *_: math.atan2(y, x))
    exp = staticmethod(lambda x, *_: math.exp(x))
    log = staticmethod(lambda x, *_: math.log(x) if x > 0 else (-math.inf if x == 0 else math.nan))
    pow = staticmethod(lambda a, b, *_: float(a) ** b)


def _object_assign(target, *srcs):
    for s in srcs:
        if s:
            for k, v in s.items():
                target[k] = v
    return target


Object = JSObject(assign=_object_assign, keys=lambda o, *_: JSArray(o.keys()))
Number = JSObject(isFinite=lambda v, *_: isinstance(v, (int, float)) and math.isfinite(v),
                  isInteger=lambda v, *_: isinstance(v, int) or (isinstance(v, float)
                                                                and v.is_integer()))


def _postinc_item(obj, k, d):
    v = obj[k]
    obj[k] = v + d
    return v


def _preinc_item(obj, k, d):
    v = obj[k] + d
    obj[k] = v
    return v


def _postinc_attr(obj, k, d):
    v = getattr(obj, k)
    setattr(obj, k, v + d)
    return v


def _preinc_attr(obj, k, d):
    v = getattr(obj, k) + d
    setattr(obj, k, v)
    return v


def _opassign_item(obj, k, fn, r):
    v = fn(obj[k], r)
    obj[k] = v
    return v


def _opassign_attr(obj, k, fn, r):
    v = fn(getattr(obj, k), r)
    setattr(obj, k, v)
    return v


def _assign_item(obj, k, v):
    obj[k] = v
    return v


def _assign_attr(obj, k, v):
    setattr(obj, k, v)
    return v


def _iter_keys(o):
    return list(o.keys()) if isinstance(o, dict) else [str(i) for i in range(len(o))]


def _get(obj, k):
    """Computed member access on any object (class instances included)."""
    if isinstance(obj, (list, array.array, dict)):
        return obj[k]
    return getattr(obj, _mangle(str(k)), None)


def _set(obj, k, v):
    if isinstance(obj, (list, array.array, dict)):
        obj[k] = v
    else:
        setattr(obj, _mangle(str(k)), v)
    return v


class JSClassBase:
    """Base of translated classes: computed member access maps to attributes."""

    def __getitem__(self, k):
        return getattr(self, _mangle(str(k)), None)

    def __setitem__(self, k, v):
        setattr(self, _mangle(str(k)), v)


def make_global() -> JSObject:
    g = JSObject()
    g["Math"] = _Math()
    g["Object"] = Object
    g["Number"] = Number
    return g


RUNTIME = {
    "JSObject": JSObject, "JSArray": JSArray, "JSError": JSError, "JSClassBase": JSClassBase,
    "Error": js_error, "TypeError": js_error, "RangeError": js_error,
    "Float32Array": Float32Array, "Float64Array": Float64Array, "Int32Array": Int32Array,
    "Uint32Array": Uint32Array, "Int16Array": Int16Array, "Uint16Array": Uint16Array,
    "Int8Array": Int8Array, "Uint8Array": Uint8Array,
    "Object": Object, "Number": Number, "Infinity": math.inf, "NaN": math.nan,
    "undefined": None, "isFinite": lambda v, *_: math.isfinite(js_tonumber(v)),
    "isNaN": lambda v, *_: js_tonumber(v) != js_tonumber(v),
    "_toint32": toint32, "_touint32": touint32, "_tonumber": js_tonumber, "_mod": js_mod,
    "_div": js_div, "_typeof": js_typeof, "_postinc_item": _postinc_item,
    "_preinc_item": _preinc_item, "_postinc_attr": _postinc_attr, "_preinc_attr": _preinc_attr,
    "_opassign_item": _opassign_item, "_opassign_attr": _opassign_attr,
    "_assign_item": _assign_item, "_assign_attr": _assign_attr, "_iter_keys": _iter_keys,
    "_get": _get, "_set": _set, "_math": math, "_sign": _sign,
}

# ============================================================================ code generation
_PY_RESERVED = set(keyword.kwlist) | {"print", "exec", "type", "id", "list", "dict", "str",
                                      "int", "float", "len", "range", "object", "super",
                                      "array", "math", "functools"}


def _mangle(name: str) -> str:
    return name + "_" if name in _PY_RESERVED else name


def _unmangle(name: str) -> str:
    if name.endswith("_") and name[:-1] in _PY_RESERVED:
        return name[:-1]
    return name


_BINOPS = {"+": "+", "-": "-", "*": "*", "**": "**", "<": "<", ">": ">", "<=": "<=",
           ">=": ">=", "===": "==", "!==": "!=", "==": "==", "!=": "!="}
_BIT = {"|": "|", "&": "&", "^": "^", "<<": "<<"}


class Scope:
    def __init__(self, parent, kind):
        self.parent = parent
        self.kind = kind          # 'func' or 'module'
        self.declared: set[str] = set()
        self.assigned: set[str] = set()


class Gen:
    def __init__(self):
        self.lines: list[str] = []
        self.n = 0
        self.loop_updates: list = []   # innermost-first stack of For update exprs (or None)
        self.scope: Scope | None = None

    def tmp(self, base="_t"):
        self.n += 1
        return f"{base}{self.n}"

    def emit(self, ind, s):
        self.lines.append("    " * ind + s)

    # ---- scope analysis (declared / assigned names per function)
    def analyse(self, body, params):
        sc = Scope(self.scope, "func")
        for p in params:
            sc.declared.add(p[1])

        def walk(node, top):
            if not isinstance(node, tuple):
                if isinstance(node, list):
                    for x in node:
                        walk(x, top)
                return
            if not node:
                return
            k = node[0]
            if k in ("FuncExpr", "Arrow") or (k == "FuncDecl" and not top):
                if k == "FuncDecl":
                    sc.declared.add(node[1])
                return
            if k == "FuncDecl":
                sc.declared.add(node[1])
                return
            if k == "Class":
                sc.declared.add(node[1])
                return
            if k == "Var":
                for target, init in node[2]:
                    for nm in _pattern_names(target):
                        sc.declared.add(nm)
                    walk(init, top)
                return
            if k in ("ForOf", "ForIn"):
                sc.declared.add(node[1])
            if k == "Try" and node[2]:
                sc.declared.add(node[2])
            if k == "Assign" and node[2][0] == "Id":
                sc.assigned.add(node[2][1])
            if k == "Update" and node[3][0] == "Id":
                sc.assigned.add(node[3][1])
            for x in node[1:]:
                walk(x, False if k in ("FuncExpr", "Arrow") else top)

        walk(body, True)
        return sc

    def nonlocals(self, sc: Scope):
        out = []
        for nm in sorted(sc.assigned - sc.declared):
            p = sc.parent
            while p is not None:
                if nm in p.declared:
                    out.append(("nonlocal" if p.kind == "func" else "global", nm))
                    break
                p = p.parent
        return out

    # ---- functions
    def func_def(self, ind, pyname, params, body, is_method=False, expr_body=False):
        sc = self.analyse(body if not expr_body else ("Return", body), params)
        outer = self.scope
        self.scope = sc
        ps = []
        if is_method:
            ps.append("this")
        rest = None
        for p in params:
            if p[0] == "rest":
                rest = _mangle(p[1])
            else:
                ps.append(f"{_mangle(p[1])}=None")
        ps.append(f"*{rest}" if rest else "*_rest")
        self.emit(ind, f"def {pyname}({', '.join(ps)}):")
        for kind, nm in self.nonlocals(sc):
            self.emit(ind + 1, f"{kind} {_mangle(nm)}")
        for p in params:
            if p[0] == "p" and p[2] is not None:
                nm = _mangle(p[1])
                self.emit(ind + 1, f"if {nm} is None: {nm} = {self.expr(p[2], ind + 1)}")
            if p[0] == "rest":
                self.emit(ind + 1, f"{_mangle(p[1])} = JSArray({_mangle(p[1])})")
        saved = self.loop_updates
        self.loop_updates = []
        if expr_body:
            self.emit(ind + 1, f"return {self.expr(body, ind + 1)}")
        else:
            self.hoist_funcs(ind + 1, body[1])
            for st in body[1]:
                self.stmt(st, ind + 1)
        self.emit(ind + 1, "pass")
        self.loop_updates = saved
        self.scope = outer

    def hoist_funcs(self, ind, stmts):
        for st in stmts:
            if st[0] == "FuncDecl":
                self.func_def(ind, _mangle(st[1]), st[2], st[3])

    # ---- statements
    def stmt(self, s, ind):
        k = s[0]
        if k == "Expr":
            self.expr_stmt(s[1], ind)
        elif k == "Var":
            for target, init in s[2]:
                val = self.expr(init, ind) if init is not None else "None"
                self.bind(target, val, ind)
        elif k == "FuncDecl":
            pass   # hoisted
        elif k == "Class":
            self.class_def(s, ind)
        elif k == "Return":
            self.emit(ind, "return" if s[1] is None else f"return {self.expr(s[1], ind)}")
        elif k == "If":
            self.emit(ind, f"if {self.cond(s[1], ind)}:")
            self.body(s[2], ind + 1)
            alt = s[3]
            while alt is not None and alt[0] == "If":
                self.emit(ind, f"elif {self.cond(alt[1], ind)}:")
                self.body(alt[2], ind + 1)
                alt = alt[3]
            if alt is not None:
                self.emit(ind, "else:")
                self.body(alt, ind + 1)
        elif k == "Block":
            self.hoist_funcs(ind, s[1])
            for st in s[1]:
                self.stmt(st, ind)
            if not s[1]:
                self.emit(ind, "pass")
        elif k == "For":
            _, init, test, update, body = s
            if init is not None:
                self.stmt(init, ind)
            self.emit(ind, "while True:")
            if test is not None:
                self.emit(ind + 1, f"if not ({self.cond(test, ind + 1)}): break")
            self.loop_updates.append(update)
            self.body(body, ind + 1)
            self.loop_updates.pop()
            if update is not None:
                self.expr_stmt(update, ind + 1)
        elif k == "While":
            self.emit(ind, f"while {self.cond(s[1], ind)}:")
            self.loop_updates.append(None)
            self.body(s[2], ind + 1)
            self.loop_updates.pop()
        elif k == "DoWhile":
            self.emit(ind, "while True:")
            self.loop_updates.append(None)
            self.body(s[1], ind + 1)
            self.loop_updates.pop()
            self.emit(ind + 1, f"if not ({self.cond(s[2], ind + 1)}): break")
        elif k in ("ForOf", "ForIn"):
            it = self.expr(s[2], ind)
            if k == "ForIn":
                it = f"_iter_keys({it})"
            self.emit(ind, f"for {_mangle(s[1])} in {it}:")
            self.loop_updates.append(None)
            self.body(s[3], ind + 1)
            self.loop_updates.pop()
        elif k == "Break":
            self.emit(ind, "break")
        elif k == "Continue":
            upd = self.loop_updates[-1] if self.loop_updates else None
            if upd is not None:
                self.expr_stmt(upd, ind)
            self.emit(ind, "continue")
        elif k == "Throw":
            self.emit(ind, f"raise {self.expr(s[1], ind)}")
        elif k == "Switch":
            self.switch(s, ind)
        elif k == "Try":
            _, blk, param, handler, fin = s
            self.emit(ind, "try:")
            self.body(blk, ind + 1)
            if handler is not None:
                self.emit(ind, "except Exception as _exc:")
                if param:
                    self.emit(ind + 1, f"{_mangle(param)} = _exc")
                self.body(handler, ind + 1)
            if fin is not None:
                self.emit(ind, "finally:")
                self.body(fin, ind + 1)
        elif k == "Empty":
            pass
        else:
            raise NotImplementedError(k)

    def body(self, s, ind):
        n0 = len(self.lines)
        self.stmt(s, ind)
        if len(self.lines) == n0:
            self.emit(ind, "pass")

    def switch(self, s, ind):
        disc = self.tmp("_sw")
        matched = self.tmp("_m")
        self.emit(ind, f"{disc} = {self.expr(s[1], ind)}")
        self.emit(ind, f"{matched} = False")
        self.emit(ind, "while True:")
        self.loop_updates.append(None)
        default_body = None
        for test, body in s[2]:
            if test is None:
                default_body = body
                continue
            self.emit(ind + 1, f"if {matched} or {disc} == {self.expr(test, ind + 1)}:")
            self.emit(ind + 2, f"{matched} = True")
            for st in body:
                self.stmt(st, ind + 2)
        if default_body is not None:
            for st in default_body:
                self.stmt(st, ind + 1)
        self.emit(ind + 1, "break")
        self.loop_updates.pop()

    def bind(self, target, val, ind):
        if target[0] == "Id":
            self.emit(ind, f"{_mangle(target[1])} = {val}")
        elif target[0] == "ObjPat":
            t = self.tmp()
            self.emit(ind, f"{t} = {val}")
            for key, local in target[1]:
                self.emit(ind, f"{_mangle(local)} = _get({t}, {key!r})")
        else:
            t = self.tmp()
            self.emit(ind, f"{t} = {val}")
            for i, nm in enumerate(target[1]):
                if nm is not None:
                    self.emit(ind, f"{_mangle(nm)} = {t}[{i}]")

    def class_def(self, s, ind):
        _, name, base, members = s
        pyname = _mangle(name)
        b = self.expr(base, ind) if base is not None else "JSClassBase"
        self.emit(ind, f"class {pyname}({b}):")
        props = {}
        for kind, static, mname, params, body in members:
            fname = "__init__" if mname == "constructor" else _mangle(mname)
            if kind in ("get", "set"):
                fname = f"_{kind}_{_mangle(mname)}"
                props.setdefault(mname, {})[kind] = fname
            if static:
                self.emit(ind + 1, "@staticmethod")
                self.func_def(ind + 1, fname, params, body, is_method=False)
            else:
                self.func_def(ind + 1, fname, params, body, is_method=True)
        for mname, acc in props.items():
            self.emit(ind + 1, f"{_mangle(mname)} = property({acc.get('get', 'None')}, "
                               f"{acc.get('set', 'None')})")
        self.emit(ind + 1, "pass")

    # ---- expressions
    def expr_stmt(self, e, ind):
        k = e[0]
        if k == "Assign":
            self.assign_stmt(e, ind)
        elif k == "Update":
            tgt = e[3]
            d = "1" if e[1] == "++" else "-1"
            self.emit(ind, f"{self.lvalue(tgt, ind)} += {d}")
        elif k == "Seq":
            for x in e[1]:
                self.expr_stmt(x, ind)
        elif k == "Str":
            pass   # 'use strict' and other directives
        else:
            self.emit(ind, self.expr(e, ind))

    def assign_stmt(self, e, ind):
        _, op, left, right = e
        if op == "=":
            targets = [left]
            r = right
            while r[0] == "Assign" and r[1] == "=":
                targets.append(r[2])
                r = r[3]
            val = self.expr(r, ind)
            lhs = " = ".join(self.lvalue(t, ind) for t in targets)
            self.emit(ind, f"{lhs} = {val}")
            return
        lv = self.lvalue(left, ind)
        rv = self.expr(right, ind)
        base = op[:-1]
        if base in ("+", "-", "*", "**"):
            self.emit(ind, f"{lv} {base}= {rv}")
        else:
            self.emit(ind, f"{lv} = {self.binop(base, lv, rv)}")

    def lvalue(self, t, ind):
        if t[0] == "Id":
            return _mangle(t[1])
        if t[0] == "Member":
            return f"{self.expr(t[1], ind)}.{_mangle(t[2])}"
        if t[0] == "Index":
            return f"{self.expr(t[1], ind)}[{self.expr(t[2], ind)}]"
        if t[0] == "Paren":
            return self.lvalue(t[1], ind)
        raise NotImplementedError(f"assignment target {t[0]}")

    def binop(self, op, a, b):
        if op in _BINOPS:
            return f"({a} {_BINOPS[op]} {b})"
        if op == "/":
            return f"_div({a}, {b})"
        if op == "%":
            return f"_mod({a}, {b})"
        if op in _BIT:
            return f"_toint32(_toint32({a}) {_BIT[op]} _toint32({b}))" if op == "<<" else \
                f"(_toint32({a}) {_BIT[op]} _toint32({b}))"
        if op == ">>":
            return f"(_toint32({a}) >> (_touint32({b}) & 31))"
        if op == ">>>":
            return f"(_touint32({a}) >> (_touint32({b}) & 31))"
        if op == "instanceof":
            return f"isinstance({a}, {b})"
        if op == "in":
            return f"({a} in {b})"
        raise NotImplementedError(op)

    def cond(self, e, ind):
        return self.expr(e, ind)

    def expr(self, e, ind):
        k = e[0]
        if k == "Num":
            v = e[1]
            if isinstance(v, float):
                return repr(v) if math.isfinite(v) else "_math.inf"
            return repr(v)
        if k == "Str":
            return repr(e[1])
        if k == "Bool":
            return "True" if e[1] else "False"
        if k == "Null":
            return "None"
        if k == "Id":
            return _mangle(e[1])
        if k == "This":
            return "this"
        if k == "Paren":
            return self.expr(e[1], ind)
        if k == "Array":
            parts = [(f"*{self.expr(x[1], ind)}" if x[0] == "Spread" else self.expr(x, ind))
                     for x in e[1]]
            return f"JSArray([{', '.join(parts)}])"
        if k == "Object":
            items = []
            for p in e[1]:
                if p[0] == "spread":
                    items.append(f"**{self.expr(p[1], ind)}")
                    continue
                _, key, val = p
                if isinstance(key, tuple):
                    kstr = f"str({self.expr(key[1], ind)})"
                else:
                    kstr = repr(str(key))
                items.append(f"{kstr}: {self.expr(val, ind)}")
            return f"JSObject({{{', '.join(items)}}})"
        if k == "Member":
            obj = self.expr(e[1], ind)
            if e[2] == "length":
                return f"{obj}.length"
            return f"{obj}.{_mangle(e[2])}"
        if k == "OptMember":
            obj = self.expr(e[1], ind)
            return f"(None if {obj} is None else {obj}.{_mangle(e[2])})"
        if k == "Index":
            obj, key = self.expr(e[1], ind), self.expr(e[2], ind)
            if e[1][0] == "This" or e[2][0] == "Str":
                return f"_get({obj}, {key})"
            return f"{obj}[{key}]"
        if k == "Call":
            callee = e[1]
            args = ", ".join((f"*{self.expr(a[1], ind)}" if a[0] == "Spread" else
                              self.expr(a, ind)) for a in e[2])
            return f"{self.expr(callee, ind)}({args})"
        if k == "New":
            args = ", ".join(self.expr(a, ind) for a in e[2])
            return f"{self.expr(e[1], ind)}({args})"
        if k == "Unary":
            op, a = e[1], e[2]
            if op == "typeof":
                if a[0] == "Id":
                    nm = _mangle(a[1])
                    return f"_typeof(globals().get({nm!r}, locals().get({nm!r})))"
                return f"_typeof({self.expr(a, ind)})"
            ax = self.expr(a, ind)
            if op == "!":
                return f"(not {ax})"
            if op == "-":
                return f"(-{ax})"
            if op == "+":
                return f"_tonumber({ax})"
            if op == "~":
                return f"(~_toint32({ax}))"
            if op == "void":
                return f"(({ax}) and None)"
            raise NotImplementedError(op)
        if k == "Bin":
            return self.binop(e[1], self.expr(e[2], ind), self.expr(e[3], ind))
        if k == "Logical":
            a, b = self.expr(e[2], ind), self.expr(e[3], ind)
            if e[1] == "||":
                return f"({a} or {b})"
            if e[1] == "&&":
                return f"({a} and {b})"
            t = self.tmp()
            return f"({b} if ({t} := {a}) is None else {t})"
        if k == "Cond":
            return f"({self.expr(e[2], ind)} if {self.cond(e[1], ind)} else {self.expr(e[3], ind)})"
        if k == "Assign":
            return self.assign_expr(e, ind)
        if k == "Update":
            return self.update_expr(e, ind)
        if k == "Seq":
            parts = [self.expr(x, ind) for x in e[1]]
            return f"({', '.join(parts)})[-1]"
        if k in ("FuncExpr",):
            name = self.tmp("_fn")
            self.func_def(ind, name, e[2], e[3])
            return name
        if k == "Arrow":
            _, params, body, is_expr = e
            name = self.tmp("_arrow")
            self.func_def(ind, name, params, body, expr_body=is_expr)
            return name
        raise NotImplementedError(k)

    def assign_expr(self, e, ind):
        _, op, left, right = e
        rv = self.expr(right, ind)
        if op == "=":
            if left[0] == "Id":
                return f"({_mangle(left[1])} := {rv})"
            if left[0] == "Index":
                return f"_assign_item({self.expr(left[1], ind)}, {self.expr(left[2], ind)}, {rv})"
            if left[0] == "Member":
                return f"_assign_attr({self.expr(left[1], ind)}, {_mangle(left[2])!r}, {rv})"
        base = op[:-1]
        fn = f"(lambda _a, _b: {self.binop(base, '_a', '_b')})"
        if left[0] == "Id":
            nm = _mangle(left[1])
            return f"({nm} := {self.binop(base, nm, rv)})"
        if left[0] == "Index":
            return f"_opassign_item({self.expr(left[1], ind)}, {self.expr(left[2], ind)}, {fn}, {rv})"
        if left[0] == "Member":
            return f"_opassign_attr({self.expr(left[1], ind)}, {_mangle(left[2])!r}, {fn}, {rv})"
        raise NotImplementedError("assignment target")

    def update_expr(self, e, ind):
        _, op, prefix, t = e
        d = "1" if op == "++" else "-1"
        if t[0] == "Id":
            nm = _mangle(t[1])
            return f"({nm} := {nm} + {d})" if prefix else f"(({nm} := {nm} + {d}) - {d})"
        if t[0] == "Index":
            f = "_preinc_item" if prefix else "_postinc_item"
            return f"{f}({self.expr(t[1], ind)}, {self.expr(t[2], ind)}, {d})"
        if t[0] == "Member":
            f = "_preinc_attr" if prefix else "_postinc_attr"
            return f"{f}({self.expr(t[1], ind)}, {_mangle(t[2])!r}, {d})"
        raise NotImplementedError("update target")


def _pattern_names(t):
    if t[0] == "Id":
        return [t[1]]
    if t[0] == "ObjPat":
        return [local for _, local in t[1]]
    return [n for n in t[1] if n is not None]


def translate(src: str) -> str:
    """JavaScript source -> Python source of a module body."""
    ast = Parser(src).program()
    g = Gen()
    top = g.analyse(("Block", ast[1]), [])
    top.kind = "module"
    g.scope = top
    g.hoist_funcs(0, ast[1])
    for st in ast[1]:
        g.stmt(st, 0)
    return "\n".join(g.lines) + "\n"


def run(sources: list[str], global_obj: JSObject | None = None) -> JSObject:
    """Execute JS sources in order against one global object (window / self)."""
    G = global_obj if global_obj is not None else make_global()
    ns = dict(RUNTIME)
    ns.update({"window": G, "self": G, "globalThis": G, "Math": G["Math"]})
    for src in sources:
        code = translate(src)
        for k, v in G.items():
            ns.setdefault(k, v)
        exec(compile(code, "<js>", "exec"), ns)
        for k, v in G.items():
            ns[k] = v
    return G
