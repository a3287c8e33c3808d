"""Rewrite the binary divisions of a user kernel's body into calls of
``ob2::div(lhs, rhs)`` (include/ops_b200_kernel.h).

``ob2::div`` is ``lhs / rhs`` for every operand pair whose quotient type is
not double; for double quotients it is a correctly rounded division by the
Newton-Raphson reciprocal and Markstein's final correction, which returns the
same bits as the IEEE quotient at one cost for every numerator, whereas
CUDA's division takes a long guarded path for zero numerators (frequent in
hydrodynamics kernels on regions at rest).  The rewrite is purely syntactic, so it must keep C's
grouping exactly: ``a * b / c`` becomes ``ob2::div(a * b, c)``, ``a / b * c``
becomes ``ob2::div(a, b) * c``, ``-a / b`` becomes ``ob2::div(-a, b)``.

The left operand of a ``/`` is the multiplicative chain before it (unary
expressions joined by binary ``*``, ``/``, ``%``), the right operand is the
unary expression after it.  Anything this scanner does not understand
(unknown casts, preprocessor lines in the body, macros whose expansion is not
a single token or one parenthesised group, ``sizeof``, templates) leaves that
division as it is: a division that is not rewritten is still an IEEE division,
so a refusal never changes a result.
"""

from __future__ import annotations

import re
from typing import Callable, Dict, List, Optional, Tuple

TOKEN_RE = re.compile(r"""
  (?P<num>0[xX][0-9a-fA-F.]+(?:[pP][+-]?\d+)?[uUlLfF]*
        |(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?[fFlLuU]*)
 |(?P<id>[A-Za-z_]\w*)
 |(?P<op>->|\+\+|--|<<=|>>=|<<|>>|<=|>=|==|!=|&&|\|\||\+=|-=|\*=|/=|%=|&=|\|=|\^=|::
        |[-+*/%<>=!~&|^?:;,.(){}\[\]#"'])
 |(?P<ws>\s+)
""", re.X)

KEYWORDS = {
    "return", "if", "else", "for", "while", "do", "switch", "case", "default", "break",
    "continue", "goto", "sizeof", "new", "delete", "throw", "typedef", "static", "const",
    "constexpr", "auto", "template", "typename", "operator", "using", "namespace", "struct",
    "class", "enum", "union", "volatile", "register", "extern", "inline", "alignof",
    "decltype", "static_assert",
}
# words a cast's parenthesised type may be made of
TYPE_WORDS = {
    "double", "float", "int", "long", "short", "char", "unsigned", "signed", "const", "bool",
    "size_t", "half", "complexd", "complexf", "int8_t", "int16_t", "int32_t", "int64_t",
    "uint8_t", "uint16_t", "uint32_t", "uint64_t", "ptrdiff_t",
}
PREFIX_OPS = {"-", "+", "!", "~", "*", "&", "++", "--"}
OPENERS = {"(": ")", "[": "]", "{": "}"}
CLOSERS = {")": "(", "]": "[", "}": "{"}


class _Fail(Exception):
    pass


def tokenize(masked: str) -> Optional[List[Tuple[str, str, int, int]]]:
    """(kind, text, start, end) of every token of comment-masked source, or
    None when a character is not part of C's token set."""
    toks = []
    pos, n = 0, len(masked)
    while pos < n:
        m = TOKEN_RE.match(masked, pos)
        if not m or m.end() == pos:
            return None
        kind = m.lastgroup
        if kind != "ws":
            toks.append((kind, m.group(), m.start(), m.end()))
        pos = m.end()
    return toks


class Macro:
    """A #define: whether its expansion is one token, one parenthesised group
    or one call (safe as a division operand), and for a function-like macro
    whether a division passed as an argument keeps its grouping when
    expanded (every use of every parameter is `(p)` or stands between
    operators that bind more loosely than `/` on its left and no postfix
    operator on its right)."""

    def __init__(self, params: Optional[List[str]], body: str):
        self.function_like = params is not None
        toks = tokenize(body)
        self.atomic = _atomic(toks)
        self.param_safe = bool(toks is not None and params is not None
                               and _param_safe(toks, set(params)))


LEFT_LOOSE = {"(", ",", "?", ":", "<", ">", "<=", ">=", "==", "!=", "&&", "||", "=", "+", "-"}
RIGHT_LOOSE = LEFT_LOOSE | {")", "*", "/", "%"}


def _param_safe(toks, params) -> bool:
    for k, t in enumerate(toks):
        if t[0] == "id" and t[1] in params:
            left = toks[k - 1][1] if k > 0 else "("
            right = toks[k + 1][1] if k + 1 < len(toks) else ")"
            if (left == "(" and right == ")") or (left in LEFT_LOOSE and right in RIGHT_LOOSE):
                continue
            return False
    return True


def macro_table(texts: List[str]) -> Dict[str, Macro]:
    """Every #define of texts, by name."""
    out: Dict[str, Macro] = {}
    for text in texts:
        joined = re.sub(r"\\\n", " ", text)
        for m in re.finditer(r"^[ \t]*#[ \t]*define[ \t]+(\w+)(\([^)]*\))?(.*)$", joined, re.M):
            body = re.sub(r"/\*.*?\*/|//.*$", "", m.group(3)).strip()
            params = None
            if m.group(2) is not None:
                params = [q.strip() for q in m.group(2)[1:-1].split(",") if q.strip()]
            out[m.group(1)] = Macro(params, body)
    return out


def _atomic(toks) -> bool:
    if toks is None:
        return False
    if not toks:
        return True
    if len(toks) == 1 and toks[0][0] in ("id", "num"):
        return True
    k0 = 1 if (toks[0][0] == "id" and len(toks) > 1 and toks[1][1] == "(") else 0
    if toks[k0][1] == "(":
        depth = 0
        for k in range(k0, len(toks)):
            t = toks[k]
            if t[1] in OPENERS:
                depth += 1
            elif t[1] in CLOSERS:
                depth -= 1
                if depth == 0:
                    return k == len(toks) - 1
    return False


class _Scan:
    def __init__(self, toks, macros: Dict[str, "Macro"]):
        self.t = toks
        self.macros = macros
        self.match: Dict[int, int] = {}
        stack = []
        for k, tk in enumerate(toks):
            if tk[1] in OPENERS:
                stack.append(k)
            elif tk[1] in CLOSERS:
                if not stack or toks[stack[-1]][1] != CLOSERS[tk[1]]:
                    raise _Fail()
                o = stack.pop()
                self.match[o] = k
                self.match[k] = o
        if stack:
            raise _Fail()

    def s(self, k: int) -> str:
        return self.t[k][1] if 0 <= k < len(self.t) else ""

    def kind(self, k: int) -> str:
        return self.t[k][0] if 0 <= k < len(self.t) else ""

    def is_name(self, k: int) -> bool:
        return self.kind(k) == "id" and self.s(k) not in KEYWORDS

    def ends_operand(self, k: int) -> bool:
        return self.is_name(k) or self.kind(k) == "num" or self.s(k) in (")", "]")

    def is_type_group(self, o: int, c: int) -> bool:
        inner = [self.s(k) for k in range(o + 1, c)]
        return bool(inner) and all(w in TYPE_WORDS or w == "*" for w in inner) \
            and any(w in TYPE_WORDS and w != "const" for w in inner)

    # -- right operand: a unary expression starting at j; returns its end --
    def unary_end(self, j: int) -> int:
        while self.s(j) in PREFIX_OPS:
            j += 1
        if self.s(j) == "(" and self.is_type_group(j, self.match[j]):
            return self.unary_end(self.match[j] + 1)
        return self.postfix_end(j)

    def postfix_end(self, j: int) -> int:
        if self.is_name(j):
            j += 1
            while self.s(j) == "::" and self.is_name(j + 1):
                j += 2
        elif self.kind(j) == "num":
            j += 1
        elif self.s(j) == "(":
            j = self.match[j] + 1
        else:
            raise _Fail()
        while True:
            if self.s(j) in ("(", "["):
                j = self.match[j] + 1
            elif self.s(j) in (".", "->") and self.is_name(j + 1):
                j += 2
            elif self.s(j) in ("++", "--"):
                raise _Fail()
            else:
                return j

    # -- left operand: the start of the unary expression ending at e ------
    def unary_start(self, e: int) -> int:
        s = self.postfix_start(e)
        while True:
            p = s - 1
            if self.s(p) in ("++", "--", "sizeof", "alignof", "new", "delete"):
                raise _Fail()  # these bind to the operand, not to the quotient
            if self.s(p) in PREFIX_OPS:
                if self.ends_operand(p - 1):
                    return s  # a binary operator: the unary expression ends here
                if self.s(p - 1) in ("++", "--"):
                    raise _Fail()
                s = p
            elif self.s(p) == ")":
                o = self.match[p]
                if not self.is_type_group(o, p):
                    raise _Fail()  # `) x` that is not a known cast
                s = o
            else:
                return s

    def postfix_start(self, e: int) -> int:
        k = e
        while True:
            t = self.s(k)
            if t in (")", "]"):
                o = self.match[k]
                if t == ")" and self.is_type_group(o, k):
                    raise _Fail()  # a cast cannot end an operand
                if self.ends_operand(o - 1):
                    k = o - 1  # call, subscript or a chained postfix
                    continue
                s = o
            elif self.is_name(k) or self.kind(k) == "num":
                s = k
                if self.kind(k) == "id" and self.s(k - 1) == "::":
                    if self.is_name(k - 2):
                        k -= 2
                        continue
                    s = k - 1  # a name in the global namespace
                    if self.ends_operand(s - 1):
                        raise _Fail()
            elif t in ("++", "--"):
                raise _Fail()
            else:
                raise _Fail()
            if self.s(s - 1) in (".", "->"):
                k = s - 2
                continue
            return s

    def chain_start(self, i: int) -> int:
        s = self.unary_start(i - 1)
        while self.s(s - 1) in ("*", "/", "%") and self.ends_operand(s - 2):
            s = self.unary_start(s - 2)
        return s

    def check_macros(self, a: int, b: int) -> None:
        """Operands may name only macros that expand to one operand, and the
        division may sit inside the arguments of a function-like macro only
        if that macro keeps the grouping of its arguments."""
        for k in range(a, b):
            m = self.macros.get(self.s(k)) if self.kind(k) == "id" else None
            if m is not None and not m.atomic:
                raise _Fail()
        for o in range(a):
            if self.s(o) == "(" and self.match[o] >= b:
                m = self.macros.get(self.s(o - 1)) if self.kind(o - 1) == "id" else None
                if m is not None and m.function_like and not m.param_safe:
                    raise _Fail()


def rewrite_divisions(body: str, mask_comments_strings: Callable[[str], str],
                      macros: Optional[Dict[str, Macro]] = None,
                      func: str = "::ob2::div") -> Tuple[str, int, int]:
    """Return (body with its divisions rewritten, rewritten count, kept
    count).  body is C/C++ source (a function body); comments are left in
    place.  mask_comments_strings(src) must blank comments and the contents of
    string and character literals, keeping every offset."""
    macros = macros or {}
    masked = mask_comments_strings(body)
    if re.search(r"^[ \t]*#", masked, re.M):
        n = len(re.findall(r"(?<![/*])/(?![/=*])", masked))
        return body, 0, n
    done = 0
    skip = 0
    while True:
        masked = mask_comments_strings(body)
        toks = tokenize(masked)
        if toks is None:
            return body, done, 0
        slashes = [k for k, t in enumerate(toks) if t[1] == "/"]
        if len(slashes) <= skip:
            return body, done, skip
        i = slashes[skip]
        try:
            sc = _Scan(toks, macros)
            a = sc.chain_start(i)
            b = sc.unary_end(i + 1)
            nxt = sc.s(b)
            if sc.kind(b) in ("id", "num") or nxt in ("(", "[", "++", "--", "{"):
                raise _Fail()
            sc.check_macros(a, b)
            if "//" in body[toks[a][2]:toks[b - 1][3]]:
                raise _Fail()  # a line comment inside an operand
        except (_Fail, KeyError):
            skip += 1
            continue
        ta, ti, ti1, tb = toks[a][2], toks[i][2], toks[i][3], toks[b - 1][3]
        body = (body[:ta] + func + "(" + body[ta:ti].rstrip() + ", " + body[ti1:tb].lstrip()
                + ")" + body[tb:])
        done += 1
