"""Restatement of pygranite's custom-expression language (TEST INFRASTRUCTURE ONLY).

The reference parses AdditionalCompute strings with cpp-peglib (an un-vendored submodule,
`.gitmodules:4-6`, commit unpinned) using the grammar in
source/granite/TrajectoryIntegrator.cpp:10-26.  This module restates that grammar as a
hand-written PEG recognizer with the same ordered-choice / no-backtrack-after-success
behaviour, builds the same AST node types (source/granite/Language.hpp:17-73), substitutes
the environment (cpp:744-768), checks tokens against the enabled features
(TrajectoryIntegrator.tpp:656-696) and flattens pre-order exactly as cpp:770-798.

Only the oracle and the tests use this; the product has its own C++ compiler to bytecode.
"""
from __future__ import annotations

import ctypes
import ctypes.util

import numpy as np

# Node types, Language.hpp:17-73
NONE, X, Y, Z, CV = 0, 1, 2, 3, 4
F0 = 5
C0 = 13
CONSTANT = 17
ADD, MUL, SUB, DIV = 18, 19, 20, 21
SQRT = 22  # SQRT..ATAN2 = 22..31 in FunctionExpression choice order
U, V, W = 33, 34, 35
IDENT = 32

FUNCTIONS = ["sqrt", "exp", "ln", "sin", "cos", "tan", "asin", "acos", "atan", "atan2"]
REGISTERS = [("x", X), ("y", Y), ("z", Z), ("cv", CV), ("u", U), ("v", V), ("w", W)]
OLD_REGISTERS = [f"f{i}" for i in range(8)] + [f"c{i}" for i in range(4)]

ERR_USER = "ERROR < USER INPUT | {} >"

_libc = ctypes.CDLL(ctypes.util.find_library("c"))
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]


def _to_float32(token: str) -> float:
    """Correctly rounded decimal -> float32, like token_to_number<float> (no double rounding)."""
    return float(_libc.strtof(token.encode(), None))


class ExprError(RuntimeError):
    pass


class Node:
    __slots__ = ("type", "value", "ident", "left", "right")

    def __init__(self, type_, value=0.0, left=None, right=None, ident=""):
        self.type = type_
        self.value = value
        self.left = left
        self.right = right
        self.ident = ident

    def __repr__(self):
        return f"Node({self.type}, {self.value}, {self.ident!r}, {self.left!r}, {self.right!r})"


class _Parser:
    """PEG recognizer for the grammar at TrajectoryIntegrator.cpp:10-26.

    %whitespace <- [ \\t]* is skipped at the start of input and after every literal/token.
    Each parse_* returns (node, new_pos) or None; ordered choice commits to the first
    alternative that succeeds.
    """

    def __init__(self, text: str):
        self.s = text
        self.n = len(text)

    def ws(self, i):
        while i < self.n and self.s[i] in " \t":
            i += 1
        return i

    def lit(self, i, word):
        if self.s.startswith(word, i):
            return self.ws(i + len(word))
        return None

    def expression(self, i):
        # OperatorExpression(A, O) <- A (O A)*  with precedence  L + -  <  L * /
        first = self.primary(i)
        if first is None:
            return None
        operands, ops = [first[0]], []
        i = first[1]
        while True:
            if i < self.n and self.s[i] in "+-*/":
                j = self.ws(i + 1)
                nxt = self.primary(j)
                if nxt is None:
                    break
                ops.append(self.s[i])
                operands.append(nxt[0])
                i = nxt[1]
            else:
                break
        return self.climb(operands, ops), i

    @staticmethod
    def climb(operands, ops):
        """Precedence climbing, both levels left-associative (cpp:21-25)."""
        prec = {"+": 1, "-": 1, "*": 2, "/": 2}
        kind = {"+": ADD, "-": SUB, "*": MUL, "/": DIV}

        def helper(lhs, idx, min_prec):
            while idx < len(ops) and prec[ops[idx]] >= min_prec:
                op = ops[idx]
                rhs = operands[idx + 1]
                idx += 1
                while idx < len(ops) and prec[ops[idx]] > prec[op]:
                    rhs, idx = helper(rhs, idx, prec[op] + 1)
                lhs = Node(kind[op], 0.0, lhs, rhs)
            return lhs, idx

        return helper(operands[0], 0, 1)[0]

    def primary(self, i):
        # '(' Expression ')' / FunctionExpression / Register / OldRegister / Identifier / Constant
        j = self.lit(i, "(")
        if j is not None:
            e = self.expression(j)
            if e is not None:
                k = self.lit(e[1], ")")
                if k is not None:
                    return e[0], k
        r = self.function(i)
        if r is not None:
            return r
        for word, t in REGISTERS:
            j = self.lit(i, word)
            if j is not None:
                return Node(t), j
        for word in OLD_REGISTERS:
            if self.s.startswith(word, i):
                raise ExprError(ERR_USER.format(
                    f"Identifier '{word}' is no longer allowed, see documentation for more information."))
        r = self.identifier(i)
        if r is not None:
            return r
        return self.constant(i)

    def function(self, i):
        for idx, name in enumerate(FUNCTIONS):
            j = self.lit(i, name)
            if j is None:
                continue
            j = self.lit(j, "(")
            if j is None:
                continue
            a = self.expression(j)
            if a is None:
                continue
            if name == "atan2":
                j = self.lit(a[1], ",")
                if j is None:
                    continue
                b = self.expression(j)
                if b is None:
                    continue
                j = self.lit(b[1], ")")
                if j is None:
                    continue
                return Node(SQRT + idx, 0.0, a[0], b[0]), j
            j = self.lit(a[1], ")")
            if j is None:
                continue
            return Node(SQRT + idx, 0.0, a[0], None), j
        return None

    def identifier(self, i):
        s = self.s
        if i < self.n and (s[i] == "_" or s[i].isascii() and s[i].isalpha()):
            j = i + 1
            while j < self.n and (s[j] == "_" or s[j].isascii() and s[j].isalnum()):
                j += 1
            return Node(IDENT, ident=s[i:j]), self.ws(j)
        return None

    def constant(self, i):
        s = self.s

        def digits(k):
            st = k
            while k < self.n and s[k].isdigit() and s[k].isascii():
                k += 1
            return k if k > st else None

        for decimal in (True, False):
            k = i
            if k < self.n and s[k] == "-":
                k += 1
            k = digits(k)
            if k is None:
                continue
            if decimal:
                if k < self.n and s[k] == ".":
                    k2 = digits(k + 1)
                    if k2 is None:
                        continue
                    k = k2
                else:
                    continue
            return Node(CONSTANT, _to_float32(s[i:k])), self.ws(k)
        return None


def parse(code: str) -> Node:
    p = _Parser(code)
    r = p.expression(p.ws(0))
    if r is None or r[1] != p.n:
        at = 0 if r is None else r[1]
        raise ExprError(ERR_USER.format(f"syntax error at column {at + 1} ( LINE: 1 COLUMN: {at + 1})"))
    return r[0]


def replace_environment(node: Node, env: dict) -> Node:
    """cpp:744-768"""
    if node.type == IDENT:
        if node.ident in env:
            node.type = env[node.ident]
            node.value = 0.0
            node.left = node.right = None
        else:
            raise ExprError(ERR_USER.format(f"Invalid identifier '{node.ident}'."))
    if node.left is not None:
        node.left = replace_environment(node.left, env)
    if node.right is not None:
        node.right = replace_environment(node.right, env)
    return node


def contains(node: Node, t: int) -> bool:
    if node.type == t:
        return True
    return (node.left is not None and contains(node.left, t)) or (
        node.right is not None and contains(node.right, t))


def flatten(node: Node | None) -> list:
    """Pre-order flat array, cpp:770-798: [type, value, left, right] per node."""
    if node is None:
        return []
    left = flatten(node.left)
    right = flatten(node.right)
    off = 1
    for e in left:
        if e[2] != -1:
            e[2] += off
        if e[3] != -1:
            e[3] += off
    off += len(left)
    for e in right:
        if e[2] != -1:
            e[2] += off
        if e[3] != -1:
            e[3] += off
    return [[node.type, node.value, 1 if node.left is not None else -1,
             off if node.right is not None else -1]] + left + right


NODE_DTYPE = np.dtype([("type", "<u4"), ("value", "<f4"), ("left", "<i4"), ("right", "<i4")])


def compile_expression(code: str, volume_names=(), constant_names=(), dim=3,
                       curvature_mode=0) -> np.ndarray:
    """parse -> replace_environment -> token checks -> flatten (tpp:656-698)."""
    env = {}
    for k, name in enumerate(list(volume_names)[:8]):
        env[name] = F0 + k
    for k, name in enumerate(list(constant_names)[:4]):
        env[name] = C0 + k
    ast = replace_environment(parse(code), env)
    nvol = min(len(volume_names), 8)
    ncon = min(len(constant_names), 4)
    if dim == 2 and contains(ast, Z):
        raise ExprError(ERR_USER.format("Compute code contains undefinded token 'z'"))
    if dim == 2 and contains(ast, W):
        raise ExprError(ERR_USER.format("Compute code contains undefinded token 'w'"))
    for k in range(7, -1, -1):
        if nvol < k + 1 and contains(ast, F0 + k):
            raise ExprError(ERR_USER.format(f"Compute code contains undefinded token 'f{k}'"))
    for k in range(4):
        if ncon < k + 1 and contains(ast, C0 + k):
            raise ExprError(ERR_USER.format(f"Compute code contains undefinded token 'c{k}'"))
    if curvature_mode != 3 and contains(ast, CV):
        raise ExprError(ERR_USER.format("Compute code contains undefinded token 'cv'"))
    flat = flatten(ast)
    arr = np.zeros(len(flat), dtype=NODE_DTYPE)
    for i, (t, v, lft, rgt) in enumerate(flat):
        arr[i] = (t, v, lft, rgt)
    return arr
