#!/usr/bin/env python3
"""Translate the reference's Rust post-processing and linking into Python.

TEST INFRASTRUCTURE ONLY (part of the oracle).  The Rust stages of the hot
path — filter_close_trackpy, prune_blobs_log, the doughnut block of
post_process, column layout and durations (src/execute_gpu.rs), the Linker
and its subnet search (src/linking.rs), circle_inds / annulus_inds
(src/kernels.rs) — cannot be compiled here (no Rust toolchain).  This
translator reads them from the reference checkout at build time, parses the
Rust subset they are written in, and emits Python that runs them with Rust's
semantics (oracle/rust_rt.py: binary32 arithmetic on numpy.float32 scalars,
truncating integer division, wrapping casts, lazy iterators, Option as
value-or-None, Err as an exception).  The output goes only to oracle/_ref/
(git-ignored): no reference source is stored in this repository.  It is the
Rust counterpart of oracle/wgsl2cpp.py, which does the same for the shaders.

What is translated is named below (ITEMS, FRAGMENTS); everything else in the
files is skipped.  Fragments are statements of a larger function
(execute_gpu's worker set-up and its duration column) wrapped in a function
whose signature this file states.

Usage: rust2py.py <reference_root> <out_dir>
"""
import keyword
import os
import re
import sys
from fractions import Fraction

import numpy as np

# ------------------------------------------------------------------ selection
ITEMS = [
    # (file, kind, name)
    ("src/kernels.rs", "fn", "circle_inds"),
    ("src/kernels.rs", "fn", "annulus_inds"),
    ("src/execute_gpu.rs", "struct", "ResultRow"),
    ("src/execute_gpu.rs", "impl", "ResultRow"),
    ("src/execute_gpu.rs", "struct", "PostProcessKernels"),
    ("src/execute_gpu.rs", "struct", "FloatMemoizer"),
    ("src/execute_gpu.rs", "impl", "FloatMemoizer"),
    ("src/execute_gpu.rs", "fn", "column_names"),
    ("src/execute_gpu.rs", "fn", "filter_close_trackpy"),
    ("src/execute_gpu.rs", "fn", "prune_blobs_log"),
    ("src/execute_gpu.rs", "fn", "post_process"),
    ("src/linking.rs", "enum", "SubsetterOutput"),
    ("src/linking.rs", "impl", "SubsetterOutput"),
    ("src/linking.rs", "enum", "SubsetterType"),
    ("src/linking.rs", "struct", "FrameSubsetter"),
    ("src/linking.rs", "impl", "FrameSubsetter"),
    ("src/linking.rs", "impl", "KdIndexTree"),
    ("src/linking.rs", "struct", "ReuseVecofVec"),
    ("src/linking.rs", "impl", "ReuseVecofVec"),
    ("src/linking.rs", "struct", "Linker"),
    ("src/linking.rs", "struct", "DurationBookkeep"),
    ("src/linking.rs", "impl", "DurationBookkeep"),
    ("src/linking.rs", "impl", "Linker"),
    ("src/linking.rs", "fn", "link"),
    ("src/linking.rs", "fn", "linker_all"),
    ("src/linking.rs", "enum", "LR"),
    ("src/linking.rs", "struct", "LRContainer"),
    ("src/linking.rs", "impl", "LRContainer"),
    ("src/linking.rs", "fn", "fill_base"),
    ("src/linking.rs", "fn", "sync_iterators"),
    ("src/linking.rs", "fn", "connect_all"),
]

# Statements of execute_gpu (src/execute_gpu.rs) run as functions.  Each is
# (file, first line regex, last line regex, wrapper head, wrapper tail): the
# source lines from the first match through the next match of the last regex
# are placed between head and tail.
FRAGMENTS = [
    # the worker thread's doughnut kernels (src/execute_gpu.rs:924-938)
    ("src/execute_gpu.rs", r"let mut kernels = if send_frame \{", r"^\s*\};\s*$",
     "fn make_kernels(tracking_params: &TrackingParams, send_frame: bool) -> Option<PostProcessKernels> {",
     "kernels }"),
    # the duration column appended after linking (src/execute_gpu.rs:1164-1181)
    ("src/execute_gpu.rs", r"let \(col_names, particle_column\) = column_names\(tracking_params\);",
     r"^\s*\};\s*$",
     "fn append_durations(output: Vec<f32>, part_durations: Option<Vec<DurationBookkeep>>, "
     "tracking_params: &TrackingParams) -> Vec<f32> {",
     "output }"),
]

TYPE_ALIASES = {"my_dtype": "f32", "float": "f32", "my_dtype_u": "u32"}
NUM_TYPES = {"f32", "f64", "u8", "u16", "u32", "u64", "usize", "i8", "i16", "i32", "i64", "isize", "bool"}

# external paths (the standard library and crates) -> runtime names
PATHS = {
    "Vec::new": "list", "Vec::with_capacity": "(lambda _n: [])", "HashMap::new": "dict", "HashSet::new": "set",
    "VecDeque::new": "rt.collections.deque", "HashSet::from_iter": "(lambda _x: set(rt.iterate(_x)))",
    "Vec::from_iter": "(lambda _x: list(rt.iterate(_x)))", "std::iter::once": "rt.once", "iter::once": "rt.once",
    "std::cmp::max_by": "rt.max_by", "std::cmp::min_by": "rt.min_by", "f32::INFINITY": "rt.INFINITY",
    "f32::NEG_INFINITY": "rt.NEG_INFINITY", "f32::NAN": "rt.NAN", "PI": "rt.PI", "std::f32::consts::PI": "rt.PI",
    "kd_tree::KdIndexTree::build_by_ordered_float": "rt.KdIndexTree.build_by_ordered_float",
    "KdIndexTree::build_by_ordered_float": "rt.KdIndexTree.build_by_ordered_float",
    "LinkingWarning::empty": "rt.LinkingWarning.empty",
    "LinkingWarning::SUBNET_FRACTION_TOO_HIGH": "rt.LinkingWarning.SUBNET_FRACTION_TOO_HIGH",
    "LinkingWarning::COMPUTATION_TOO_HEAVY": "rt.LinkingWarning.COMPUTATION_TOO_HEAVY",
    "ndarray::Ix2": "rt.Ix2", "ArrayView::from_shape": "rt.ArrayView.from_shape",
    "Array::zeros": "(lambda _s: rt.np.zeros(_s, rt.np.float32))", "Axis": "(lambda _a: _a)",
    "N::to_usize": "(lambda: 2)", "Box::new": "(lambda _x: _x)", "Some": "(lambda _x: _x)",
    "Ok": "(lambda _x: _x)", "Err": "rt.err", "None": "None",
    "kernels::circle_inds": "circle_inds", "kernels::annulus_inds": "annulus_inds",
}
ENUM_PREFIXES = {"Ordering": "rt.Ordering", "std::cmp::Ordering": "rt.Ordering",
                 "std::sync::atomic::Ordering": "rt.Ordering"}
ERROR_PREFIXES = ("Error", "crate::error::Error")
IDENTITY_METHODS = {"into_slice"}


class TranslateError(Exception):
    pass


# ------------------------------------------------------------------ lexer
TOKEN_RE = re.compile(r"""
 (?P<ws>\s+)|(?P<lc>//[^\n]*)|(?P<bc>/\*.*?\*/)|
 (?P<str>b?"(?:\\.|[^"\\])*")|
 (?P<chr>'(?:\\.|[^'\\])')|
 (?P<life>'[A-Za-z_][A-Za-z0-9_]*)|
 (?P<num>\d[\d_]*\.(?![.\w])|\d[\d_]*(?:\.\d[\d_]*)?(?:[eE][+-]?\d+)?(?:f32|f64|u8|u16|u32|u64|usize|i8|i16|i32|i64|isize)?)|
 (?P<id>[A-Za-z_][A-Za-z0-9_]*)|
 (?P<op>::|->|=>|==|!=|<=|>=|&&|\|\||\+=|-=|\*=|/=|%=|\|=|&=|\^=|\.\.=|\.\.\.|\.\.|[-+*/%=<>!&|^.,;:\#?@(){}\[\]$~])
""", re.S | re.X)


class Tok:
    __slots__ = ("kind", "val", "line")

    def __init__(self, kind, val, line):
        self.kind, self.val, self.line = kind, val, line

    def __repr__(self):
        return "%s:%r@%d" % (self.kind, self.val, self.line)


def lex(src):
    toks, pos, line = [], 0, 1
    while pos < len(src):
        m = TOKEN_RE.match(src, pos)
        if not m:
            raise TranslateError("lex error at line %d: %r" % (line, src[pos:pos + 30]))
        kind = m.lastgroup
        val = m.group(kind)
        if kind not in ("ws", "lc", "bc"):
            toks.append(Tok(kind, val, line))
        line += val.count("\n")
        pos = m.end()
    toks.append(Tok("eof", "", line))
    return toks


# ------------------------------------------------------------------ parser
BLOCKLIKE = ("if", "match", "for", "while", "loop", "block", "unsafe")
BINOPS = {"||": 1, "&&": 2, "==": 3, "!=": 3, "<": 3, ">": 3, "<=": 3, ">=": 3, "|": 4, "^": 5, "&": 6,
          "<<": 7, ">>": 7, "+": 8, "-": 8, "*": 9, "/": 9, "%": 9}
ASSIGN_OPS = ("=", "+=", "-=", "*=", "/=", "%=", "|=", "&=", "^=")


class Parser:
    def __init__(self, toks, want=None):
        self.t = toks
        self.i = 0
        # want(kind, name) -> bool: items not wanted are skipped unparsed
        self.want = want or (lambda kind, name: True)

    # --- token helpers
    def peek(self, k=0):
        return self.t[min(self.i + k, len(self.t) - 1)]

    def at(self, *vals):
        return self.peek().val in vals and self.peek().kind in ("op", "id")

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def expect(self, val):
        tok = self.next()
        if tok.val != val:
            raise TranslateError("line %d: expected %r, got %r" % (tok.line, val, tok.val))
        return tok

    def ident(self):
        tok = self.next()
        if tok.kind != "id":
            raise TranslateError("line %d: expected identifier, got %r" % (tok.line, tok.val))
        return tok.val

    def skip_group(self):
        """Skip a balanced (...), [...] or {...} group starting at the current token."""
        open_ = self.next().val
        close = {"(": ")", "[": "]", "{": "}"}[open_]
        depth = 1
        while depth:
            tok = self.next()
            if tok.kind == "eof":
                raise TranslateError("unbalanced group")
            if tok.val in ("(", "[", "{"):
                depth += 1
            elif tok.val in (")", "]", "}"):
                depth -= 1
        return close

    def skip_generics(self):
        """Skip <...> (the current token is '<'), nesting on < > ( ) [ ]."""
        depth = 0
        while True:
            tok = self.next()
            if tok.val == "<":
                depth += 1
            elif tok.val == ">":
                depth -= 1
                if depth == 0:
                    return
            elif tok.val in ("(", "["):
                self.i -= 1
                self.skip_group()
            elif tok.kind == "eof":
                raise TranslateError("unbalanced generics")

    def skip_attrs(self):
        while self.at("#"):
            self.next()
            if self.at("!"):
                self.next()
            self.skip_group()

    def skip_vis(self):
        if self.at("pub"):
            self.next()
            if self.at("("):
                self.skip_group()

    def skip_where(self):
        if self.at("where"):
            while not self.at("{", ";"):
                if self.at("<"):
                    self.skip_generics()
                elif self.at("(", "["):
                    self.skip_group()
                else:
                    self.next()

    # --- types (kept as text; only casts and defaults look at them)
    def parse_type(self):
        if self.at("&"):
            self.next()
            if self.peek().kind == "life":
                self.next()
            if self.at("mut"):
                self.next()
            return "&" + self.parse_type()
        if self.at("&&"):
            self.next()
            return "&&" + self.parse_type()
        if self.at("("):
            self.next()
            parts = []
            while not self.at(")"):
                parts.append(self.parse_type())
                if self.at(","):
                    self.next()
            self.next()
            return "(" + ",".join(parts) + ")"
        if self.at("["):
            self.next()
            inner = self.parse_type()
            if self.at(";"):
                self.next()
                self.parse_expr()
            self.expect("]")
            return "[" + inner + "]"
        if self.at("impl", "dyn"):
            self.next()
            t = self.parse_type()
            while self.at("+"):
                self.next()
                if self.peek().kind == "life":
                    self.next()
                else:
                    self.parse_type()
            return t
        if self.at("fn", "Fn", "FnMut", "FnOnce") and self.peek(1).val == "(":
            name = self.next().val
            self.skip_group()
            if self.at("->"):
                self.next()
                self.parse_type()
            return name
        if self.at("<"):
            self.skip_generics()
            while self.at("::"):
                self.next()
                self.ident()
            return "_qualified"
        if self.at("_", "!"):
            self.next()
            return "_"
        if self.peek().kind == "life":
            self.next()
            return "'"
        segs = []
        while True:
            segs.append(self.ident())
            if self.at("<"):
                self.skip_generics()
            if self.at("(") and segs[-1] in ("Fn", "FnMut", "FnOnce"):
                self.skip_group()
                if self.at("->"):
                    self.next()
                    self.parse_type()
            if self.at("::"):
                self.next()
                continue
            break
        return "::".join(segs)

    # --- items
    def parse_items(self):
        items = []
        while self.peek().kind != "eof":
            self.skip_attrs()
            self.skip_vis()
            tok = self.peek()
            if tok.val == "use":
                while not self.at(";"):
                    if self.at("{"):
                        self.skip_group()
                    else:
                        self.next()
                self.next()
            elif tok.val in ("fn", "const", "unsafe", "async") and (tok.val == "fn" or self.peek(1).val == "fn"):
                if tok.val != "fn":
                    self.next()
                if self.want("fn", self.peek(1).val):
                    items.append(self.parse_fn())
                else:
                    while not self.at("{"):
                        if self.at("(", "["):
                            self.skip_group()
                        elif self.at("<"):
                            self.skip_generics()
                        else:
                            self.next()
                    self.skip_group()
            elif tok.val == "struct":
                items.append(self.parse_struct())
            elif tok.val == "enum":
                items.append(self.parse_enum())
            elif tok.val == "impl":
                items.append(self.parse_impl())
            elif tok.val in ("type", "const", "static"):
                while not self.at(";"):
                    if self.at("{", "(", "["):
                        self.skip_group()
                    else:
                        self.next()
                self.next()
            elif tok.val in ("trait", "mod"):
                while not self.at("{"):
                    if self.at("<"):
                        self.skip_generics()
                    else:
                        self.next()
                self.skip_group()
            elif tok.kind == "id" and self.peek(1).val == "!":
                self.next()
                self.next()
                self.skip_group()
            else:
                raise TranslateError("line %d: unexpected item token %r" % (tok.line, tok.val))
        return items

    def parse_fn(self):
        self.expect("fn")
        name = self.ident()
        if self.at("<"):
            self.skip_generics()
        self.expect("(")
        params, self_kind = [], None
        while not self.at(")"):
            self.skip_attrs()
            if self.at("self") or (self.at("&") and self.peek(1).val in ("self", "mut")
                                   and (self.peek(1).val == "self" or self.peek(2).val == "self")) or \
                    (self.at("mut") and self.peek(1).val == "self"):
                while not self.at(",", ")"):
                    self.next()
                self_kind = "self"
            else:
                pat = self.parse_pat(allow_or=False)
                self.expect(":")
                ty = self.parse_type()
                params.append((pat, ty))
            if self.at(","):
                self.next()
        self.next()
        ret = None
        if self.at("->"):
            self.next()
            ret = self.parse_type()
        self.skip_where()
        body = self.parse_block()
        return ("fn", name, params, self_kind, body, ret)

    def parse_struct(self):
        self.expect("struct")
        name = self.ident()
        if self.at("<"):
            self.skip_generics()
        self.skip_where()
        fields = []
        if self.at("{"):
            self.next()
            while not self.at("}"):
                self.skip_attrs()
                self.skip_vis()
                fname = self.ident()
                self.expect(":")
                fields.append((fname, self.parse_type()))
                if self.at(","):
                    self.next()
            self.next()
        elif self.at("("):
            self.skip_group()
            self.expect(";")
        else:
            self.expect(";")
        return ("struct", name, fields)

    def parse_enum(self):
        self.expect("enum")
        name = self.ident()
        if self.at("<"):
            self.skip_generics()
        self.expect("{")
        variants = []
        while not self.at("}"):
            self.skip_attrs()
            vname = self.ident()
            kind = "unit"
            if self.at("("):
                self.skip_group()
                kind = "tuple"
            elif self.at("{"):
                self.skip_group()
                kind = "struct"
            if self.at("="):
                self.next()
                self.parse_expr()
            variants.append((vname, kind))
            if self.at(","):
                self.next()
        self.next()
        return ("enum", name, variants)

    def parse_impl(self):
        self.expect("impl")
        if self.at("<"):
            self.skip_generics()
        first = self.parse_type()
        trait, target = None, first
        if self.at("for"):
            self.next()
            trait, target = first, self.parse_type()
        self.skip_where()
        if not self.want("impl", target.split("::")[-1]):
            self.skip_group()
            return ("impl", target.split("::")[-1], trait, [])
        self.expect("{")
        fns = []
        while not self.at("}"):
            self.skip_attrs()
            self.skip_vis()
            if self.at("type", "const"):
                while not self.at(";"):
                    self.next()
                self.next()
            elif self.at("fn"):
                fns.append(self.parse_fn())
            else:
                raise TranslateError("line %d: unexpected impl member %r" % (self.peek().line, self.peek().val))
        self.next()
        return ("impl", target.split("::")[-1], trait, fns)

    # --- blocks and statements
    def parse_block(self):
        self.expect("{")
        stmts, tail = [], None
        while not self.at("}"):
            self.skip_attrs()
            if self.at(";"):
                self.next()
                continue
            if self.at("let"):
                self.next()
                pat = self.parse_pat(allow_or=False)
                ty = None
                if self.at(":"):
                    self.next()
                    ty = self.parse_type()
                init = None
                if self.at("="):
                    self.next()
                    init = self.parse_expr()
                if self.at("else"):
                    # let-else: the else block diverges when the pattern fails
                    self.next()
                    els = self.parse_block()
                    self.expect(";")
                    stmts.append(("letelse", pat, init, els))
                    continue
                self.expect(";")
                stmts.append(("let", pat, init, ty))
                continue
            if self.at("fn") or (self.at("pub") and self.peek(1).val == "fn"):
                self.skip_vis()
                stmts.append(("item", self.parse_fn()))
                continue
            if self.at("use"):
                while not self.at(";"):
                    self.next()
                self.next()
                continue
            if self.at("if", "match", "loop", "while", "for", "{") or (self.at("unsafe") and self.peek(1).val == "{"):
                # a block-like expression statement ends at its closing brace
                e = self.parse_primary(False)
                if self.at(".", "?"):
                    self.i -= 0
                    e = self.parse_postfix_from(e)
                    while self.peek().kind == "op" and self.peek().val in BINOPS:
                        raise TranslateError("line %d: binary operator after a block statement" % self.peek().line)
            else:
                e = self.parse_expr()
            if self.at(";"):
                self.next()
                stmts.append(("expr", e, True))
            elif self.at("}"):
                tail = e
            elif e[0] in BLOCKLIKE:
                stmts.append(("expr", e, False))
            else:
                raise TranslateError("line %d: expected ';' after expression, got %r" % (self.peek().line,
                                                                                        self.peek().val))
        self.next()
        return ("block", stmts, tail)

    # --- expressions
    def parse_expr(self, ns=False):
        return self.parse_assign(ns)

    def parse_assign(self, ns):
        lhs = self.parse_range(ns)
        if self.peek().kind == "op" and self.peek().val in ASSIGN_OPS:
            op = self.next().val
            rhs = self.parse_assign(ns)
            return ("assign", op, lhs, rhs)
        return lhs

    def _range_end_follows(self):
        tok = self.peek()
        return not (tok.val in (")", "]", "}", ",", ";", "=>") or (tok.val == "{" and True))

    def parse_range(self, ns):
        if self.at("..", "..="):
            incl = self.next().val == "..="
            hi = self.parse_bin(0, ns) if self._range_end_follows() else None
            return ("range", None, hi, incl)
        lo = self.parse_bin(0, ns)
        if self.at("..", "..="):
            incl = self.next().val == "..="
            hi = self.parse_bin(0, ns) if self._range_end_follows() else None
            return ("range", lo, hi, incl)
        return lo

    def parse_bin(self, minp, ns):
        lhs = self.parse_cast(ns)
        while True:
            tok = self.peek()
            op = tok.val if tok.kind == "op" else None
            if op in (">",) and self.peek(1).val == ">" and self.peek(1).kind == "op":
                op = ">>"
            if op is None or op not in BINOPS or BINOPS[op] <= minp and not (BINOPS.get(op, 0) > minp):
                break
            p = BINOPS[op]
            if p <= minp:
                break
            self.next()
            if op == ">>":
                self.next()
            rhs = self.parse_bin(p, ns)
            lhs = ("binary", op, lhs, rhs)
        return lhs

    def parse_cast(self, ns):
        e = self.parse_unary(ns)
        while self.at("as"):
            self.next()
            e = ("cast", e, self.parse_type())
        return e

    def parse_unary(self, ns):
        if self.at("-"):
            self.next()
            return ("unary", "-", self.parse_unary(ns))
        if self.at("!"):
            self.next()
            return ("unary", "!", self.parse_unary(ns))
        if self.at("*"):
            self.next()
            return ("unary", "*", self.parse_unary(ns))
        if self.at("&&"):
            self.next()
            if self.at("mut"):
                self.next()
            return ("unary", "&", ("unary", "&", self.parse_unary(ns)))
        if self.at("&"):
            self.next()
            if self.at("mut"):
                self.next()
                return ("unary", "&mut", self.parse_unary(ns))
            return ("unary", "&", self.parse_unary(ns))
        return self.parse_postfix(ns)

    def parse_postfix(self, ns):
        return self.parse_postfix_from(self.parse_primary(ns))

    def parse_postfix_from(self, e):
        while True:
            if self.at("?"):
                self.next()
                e = ("try", e)
            elif self.at("."):
                self.next()
                tok = self.next()
                if tok.kind == "num":
                    parts = tok.val.split(".")
                    for part in parts:
                        if part:
                            e = ("field", e, int(part))
                    continue
                name = tok.val
                if self.at("::"):
                    self.next()
                    self.skip_generics()
                if self.at("("):
                    e = ("mcall", e, name, self.parse_args())
                else:
                    e = ("field", e, name)
            elif self.at("("):
                e = ("call", e, self.parse_args())
            elif self.at("["):
                self.next()
                idx = self.parse_expr()
                self.expect("]")
                e = ("index", e, idx)
            else:
                return e

    def parse_args(self):
        self.expect("(")
        args = []
        while not self.at(")"):
            args.append(self.parse_expr())
            if self.at(","):
                self.next()
        self.next()
        return args

    def parse_if(self):
        self.expect("if")
        if self.at("let"):
            self.next()
            pat = self.parse_pat(allow_or=True)
            self.expect("=")
            cond = ("let", pat, self.parse_expr(ns=True))
        else:
            cond = self.parse_expr(ns=True)
        then = self.parse_block()
        els = None
        if self.at("else"):
            self.next()
            els = self.parse_if() if self.at("if") else self.parse_block()
        return ("if", cond, then, els)

    def parse_closure(self):
        if self.at("move"):
            self.next()
        params = []
        if self.at("||"):
            self.next()
        else:
            self.expect("|")
            while not self.at("|"):
                pat = self.parse_pat(allow_or=False)
                if self.at(":"):
                    self.next()
                    self.parse_type()
                params.append(pat)
                if self.at(","):
                    self.next()
            self.next()
        if self.at("->"):
            self.next()
            self.parse_type()
            body = self.parse_block()
        else:
            body = self.parse_expr()
        return ("closure", params, body)

    def parse_macro(self, name):
        self.expect("!")
        if name == "vec":
            open_ = self.next().val
            close = {"[": "]", "(": ")", "{": "}"}[open_]
            elems = []
            if self.at(close):
                self.next()
                return ("array", elems)
            first = self.parse_expr()
            if self.at(";"):
                self.next()
                n = self.parse_expr()
                self.expect(close)
                return ("vec_rep", first, n)
            elems.append(first)
            while self.at(","):
                self.next()
                if self.at(close):
                    break
                elems.append(self.parse_expr())
            self.expect(close)
            return ("array", elems)
        if name in ("panic", "unreachable", "todo", "unimplemented"):
            self.skip_group()
            return ("panic", name)
        if name in ("println", "print", "eprintln", "eprint", "dbg", "debug_assert"):
            self.skip_group()
            return ("unit",)
        if name in ("s", "format", "matches", "write", "writeln"):
            self.skip_group()
            return ("panic", "unsupported macro %s!" % name)
        if name == "assert":
            self.expect("(")
            e = self.parse_expr()
            while not self.at(")"):
                self.next()
            self.next()
            return ("assert", e)
        raise TranslateError("line %d: unsupported macro %s!" % (self.peek().line, name))

    def parse_path(self):
        segs = []
        if self.at("<"):
            # qualified path <T as Trait>::name
            start = self.i
            self.skip_generics()
            segs.append("".join(t.val for t in self.t[start:self.i]))
            self.expect("::")
        while True:
            segs.append(self.ident())
            if self.at("::"):
                if self.peek(1).val == "<":
                    self.next()
                    self.skip_generics()
                    if not self.at("::"):
                        break
                    self.next()
                    continue
                self.next()
                continue
            break
        return segs

    def parse_primary(self, ns):
        tok = self.peek()
        if tok.kind == "num":
            self.next()
            return ("lit", "num", tok.val)
        if tok.kind == "str":
            self.next()
            return ("lit", "str", tok.val)
        if tok.kind == "chr":
            self.next()
            return ("lit", "chr", tok.val)
        v = tok.val
        if v in ("true", "false") and tok.kind == "id":
            self.next()
            return ("lit", "bool", v)
        if v == "(":
            self.next()
            if self.at(")"):
                self.next()
                return ("unit",)
            first = self.parse_expr()
            if self.at(")"):
                self.next()
                return ("paren", first)
            elems = [first]
            while self.at(","):
                self.next()
                if self.at(")"):
                    break
                elems.append(self.parse_expr())
            self.expect(")")
            return ("tuple", elems)
        if v == "[":
            self.next()
            if self.at("]"):
                self.next()
                return ("array", [])
            first = self.parse_expr()
            if self.at(";"):
                self.next()
                n = self.parse_expr()
                self.expect("]")
                return ("vec_rep", first, n)
            elems = [first]
            while self.at(","):
                self.next()
                if self.at("]"):
                    break
                elems.append(self.parse_expr())
            self.expect("]")
            return ("array", elems)
        if v == "{":
            return self.parse_block()
        if v == "unsafe" and self.peek(1).val == "{":
            self.next()
            return self.parse_block()
        if v == "if":
            return self.parse_if()
        if v == "match":
            self.next()
            scrut = self.parse_expr(ns=True)
            self.expect("{")
            arms = []
            while not self.at("}"):
                pat = self.parse_pat(allow_or=True)
                guard = None
                if self.at("if"):
                    self.next()
                    guard = self.parse_expr()
                self.expect("=>")
                # a block body ends the arm: `{ .. } (a, b) => ..` is the next arm
                body = self.parse_block() if self.at("{") else self.parse_expr()
                if self.at(","):
                    self.next()
                arms.append((pat, guard, body))
            self.next()
            return ("match", scrut, arms)
        if v == "for":
            self.next()
            pat = self.parse_pat(allow_or=False)
            self.expect("in")
            it = self.parse_expr(ns=True)
            return ("for", pat, it, self.parse_block())
        if v == "while":
            self.next()
            if self.at("let"):
                self.next()
                pat = self.parse_pat(allow_or=True)
                self.expect("=")
                cond = ("let", pat, self.parse_expr(ns=True))
            else:
                cond = self.parse_expr(ns=True)
            return ("while", cond, self.parse_block())
        if v == "loop":
            self.next()
            return ("loop", self.parse_block())
        if v in ("return", "break"):
            self.next()
            val = None
            if not self.at(";", "}", ")", ","):
                val = self.parse_expr()
            return (v, val)
        if v == "continue":
            self.next()
            return ("continue",)
        if v in ("|", "||", "move"):
            return self.parse_closure()
        if tok.kind == "id" or v == "<":
            segs = self.parse_path()
            if self.at("!") and len(segs) == 1 and self.peek(1).val in ("(", "[", "{"):
                return self.parse_macro(segs[0])
            if self.at("{") and not ns and (segs[-1][:1].isupper() or segs[-1] == "Self"):
                return self.parse_struct_lit(segs)
            return ("path", segs)
        raise TranslateError("line %d: unexpected token %r" % (tok.line, v))

    def parse_struct_lit(self, segs):
        self.expect("{")
        fields, base = [], None
        while not self.at("}"):
            if self.at(".."):
                self.next()
                base = self.parse_expr()
                continue
            name = self.ident()
            if self.at(":"):
                self.next()
                fields.append((name, self.parse_expr()))
            else:
                fields.append((name, ("path", [name])))
            if self.at(","):
                self.next()
        self.next()
        return ("struct", segs, fields, base)

    # --- patterns
    def parse_pat(self, allow_or=True):
        if allow_or and self.at("|"):
            self.next()
        p = self.parse_pat1()
        if allow_or and self.at("|"):
            alts = [p]
            while self.at("|"):
                self.next()
                alts.append(self.parse_pat1())
            return ("or", alts)
        return p

    def parse_pat_list(self, close):
        pats = []
        while not self.at(close):
            if self.at(".."):
                self.next()
                pats.append(("rest",))
            else:
                pats.append(self.parse_pat(allow_or=True))
            if self.at(","):
                self.next()
        self.next()
        return pats

    def parse_pat1(self):
        tok = self.peek()
        v = tok.val
        if v == "_" and tok.kind == "id":
            self.next()
            return ("wild",)
        if v in ("&", "&&"):
            self.next()
            if self.at("mut"):
                self.next()
            inner = self.parse_pat1()
            return ("ref", ("ref", inner) if v == "&&" else inner)
        if v == "(":
            self.next()
            return ("ptuple", self.parse_pat_list(")"))
        if v == "[":
            self.next()
            return ("pslice", self.parse_pat_list("]"))
        if tok.kind in ("num", "str", "chr") or (v == "-" and self.peek(1).kind == "num"):
            neg = False
            if v == "-":
                self.next()
                neg = True
            lit = self.next()
            return ("plit", ("lit", "num" if lit.kind == "num" else lit.kind, ("-" if neg else "") + lit.val))
        if v in ("true", "false"):
            self.next()
            return ("plit", ("lit", "bool", v))
        if v in ("ref", "mut"):
            self.next()
            if self.at("mut"):
                self.next()
            return ("bind", self.ident(), None)
        segs = self.parse_path()
        if self.at("("):
            self.next()
            return ("ptstruct", segs, self.parse_pat_list(")"))
        if self.at("{"):
            self.next()
            fields, rest = [], False
            while not self.at("}"):
                if self.at(".."):
                    self.next()
                    rest = True
                    continue
                if self.at("ref", "mut"):
                    self.next()
                    if self.at("mut"):
                        self.next()
                fname = self.ident()
                if self.at(":"):
                    self.next()
                    fields.append((fname, self.parse_pat(allow_or=True)))
                else:
                    fields.append((fname, ("bind", fname, None)))
                if self.at(","):
                    self.next()
            self.next()
            return ("pstruct", segs, fields, rest)
        if self.at("@"):
            self.next()
            return ("bind", segs[0], self.parse_pat1())
        if len(segs) == 1 and segs[0] not in ("None",):
            return ("bind", segs[0], None)
        return ("ppath", segs)


# ------------------------------------------------------------------ emitter
PY_RESERVED = set(keyword.kwlist) | {"rt", "np", "self_"}


def f32_literal(text):
    """The binary32 value nearest the decimal literal (ties to even)."""
    q = Fraction(text)
    x = np.float32(float(q))
    best = x
    for cand in (np.nextafter(x, np.float32(-np.inf)), np.nextafter(x, np.float32(np.inf))):
        d_best, d_c = abs(Fraction(float(best)) - q), abs(Fraction(float(cand)) - q)
        if d_c < d_best or (d_c == d_best and int(np.array(cand).view(np.uint32)) % 2 == 0):
            best = cand
    return float(best)


def walk(node, fn):
    """Apply fn to every tuple node of an AST (pre-order)."""
    if isinstance(node, tuple):
        fn(node)
        for c in node:
            walk(c, fn)
    elif isinstance(node, list):
        for c in node:
            walk(c, fn)


class FnInfo:
    def __init__(self, name, params, deref):
        self.name, self.params, self.deref = name, params, deref


class Emitter:
    def __init__(self):
        self.lines = []
        self.ind = 0
        self.tmp = 0
        self.scopes = []          # list of dict rust name -> python name
        self.refs = set()         # python names holding Cell / AttrRef (deref with .v)
        self.alias = {}           # python name -> expression (iter_mut element places)
        self.globals = set()
        self.structs = {}         # name -> fields
        self.enums = {}           # name -> variants
        self.fns = {}             # name -> FnInfo
        self.cls = None           # class being emitted
        self.used = set()

    # --- output
    def emit(self, line):
        self.lines.append("    " * self.ind + line)

    def temp(self, base="_t"):
        self.tmp += 1
        return "%s%d" % (base, self.tmp)

    # --- scopes
    def push(self):
        self.scopes.append({})

    def pop(self):
        self.scopes.pop()

    def lookup(self, name):
        for sc in reversed(self.scopes):
            if name in sc:
                return sc[name]
        return None

    def bind(self, name):
        """A Python name for a new Rust binding.  Rebinding in the same scope
        reuses the name; a binding that shadows one of an enclosing scope gets
        a fresh name, so the outer value is intact when the block ends."""
        base = name + "_" if name in PY_RESERVED else name
        cur = self.scopes[-1]
        if name in cur:
            py = cur[name]
        elif any(name in sc for sc in self.scopes[:-1]) or base in self.taken():
            k = 2
            while "%s_%d" % (base, k) in self.used or "%s_%d" % (base, k) in self.taken():
                k += 1
            py = "%s_%d" % (base, k)
        else:
            py = base
        self.used.add(py)
        cur[name] = py
        self.refs.discard(py)
        self.alias.pop(py, None)
        return py

    def taken(self):
        """Python names visible from the current scope (they must not be reused)."""
        out = set()
        for sc in self.scopes[:-1]:
            out.update(sc.values())
        return out

    # --- patterns
    def pat_simple(self, p):
        """A Python assignment target for a pattern made of bindings, _ and tuples, or None."""
        if p[0] == "bind" and p[2] is None:
            return self.bind(p[1])
        if p[0] == "wild":
            return "_"
        if p[0] == "ref":
            return self.pat_simple(p[1])
        if p[0] == "ptuple" and all(q[0] != "rest" for q in p[1]):
            parts = [self.pat_simple(q) for q in p[1]]
            if any(x is None for x in parts):
                return None
            return "(" + ", ".join(parts) + ("," if len(parts) == 1 else "") + ")"
        return None

    def pat_test(self, p, acc):
        """(condition, [(rust name, accessor)]) for matching pattern p against accessor acc."""
        k = p[0]
        if k == "wild" or k == "rest":
            return "True", []
        if k == "bind":
            if p[2] is None:
                return "True", [(p[1], acc)]
            c, b = self.pat_test(p[2], acc)
            return c, b + [(p[1], acc)]
        if k == "ref":
            return self.pat_test(p[1], acc)
        if k in ("ptuple", "pslice"):
            conds, binds = [], []
            items = p[1]
            if any(q[0] == "rest" for q in items):
                r = [i for i, q in enumerate(items) if q[0] == "rest"][0]
                head, tail = items[:r], items[r + 1:]
                idx = [(str(i), q) for i, q in enumerate(head)] + [("-%d" % (len(tail) - i), q)
                                                                  for i, q in enumerate(tail)]
            else:
                idx = [(str(i), q) for i, q in enumerate(items)]
                if k == "pslice":
                    conds.append("len(%s) == %d" % (acc, len(items)))
            for i, q in idx:
                c, b = self.pat_test(q, "%s[%s]" % (acc, i))
                if c != "True":
                    conds.append(c)
                binds += b
            return (" and ".join("(%s)" % c for c in conds) if conds else "True"), binds
        if k == "plit":
            return "%s == %s" % (acc, self.expr(p[1])), []
        if k == "ppath":
            last = p[1][-1]
            if last == "None":
                return "%s is None" % acc, []
            return "rt.tag_is(%s, %r)" % (acc, last), []
        if k == "ptstruct":
            last = p[1][-1]
            subs = p[2]
            if last == "Some":
                c, b = self.pat_test(subs[0], acc)
                return ("%s is not None" % acc) + ("" if c == "True" else " and (%s)" % c), b
            if last == "Ok":
                return self.pat_test(subs[0], acc)
            if last == "Err":
                return "False", []
            conds, binds = ["rt.tag_is(%s, %r)" % (acc, last)], []
            for i, q in enumerate(subs):
                c, b = self.pat_test(q, "%s.vals[%d]" % (acc, i))
                if c != "True":
                    conds.append(c)
                binds += b
            return " and ".join("(%s)" % c for c in conds), binds
        if k == "pstruct":
            last = p[1][-1]
            conds, binds = [], []
            if last not in self.structs and last != "Self":
                conds.append("rt.tag_is(%s, %r)" % (acc, last))
            for fname, q in p[2]:
                c, b = self.pat_test(q, "%s.%s" % (acc, fname))
                if c != "True":
                    conds.append(c)
                binds += b
            return (" and ".join("(%s)" % c for c in conds) if conds else "True"), binds
        if k == "or":
            # alternatives that match an Err never match (errors are raised)
            alts = [self.pat_test(q, acc) for q in p[1]]
            alts = [(c, b) for c, b in alts if c != "False" and "(False)" not in c]
            if not alts:
                return "False", []
            if len(alts) == 1:
                return alts[0]
            if any(b for _, b in alts):
                raise TranslateError("bindings inside an or-pattern")
            return " or ".join("(%s)" % c for c, _ in alts), []
        raise TranslateError("pattern %r" % (p,))

    def bind_all(self, binds):
        for name, acc in binds:
            py = self.bind(name)
            self.emit("%s = %s" % (py, acc))

    # --- expressions
    def path_expr(self, segs):
        if len(segs) == 1:
            n = segs[0]
            if n == "self":
                return "self"
            py = self.lookup(n)
            if py is not None:
                if py in self.alias:
                    return self.alias[py]
                return py
            if n in PATHS:
                return PATHS[n]
            if n in self.globals:
                return n
            if n == "Self":
                return self.cls
            raise TranslateError("unknown name %s" % n)
        full = "::".join(segs)
        if full in PATHS:
            return PATHS[full]
        head, last = "::".join(segs[:-1]), segs[-1]
        if head in ENUM_PREFIXES:
            return "%s.%s" % (ENUM_PREFIXES[head], last)
        if head in ERROR_PREFIXES:
            return "rt.Error(%r)" % last
        if head == "Self":
            return "%s.%s" % (self.cls, last)
        if head.startswith("<") and last == "zero":
            return "(lambda: rt.F32(0.0))"
        if segs[-2] in self.structs or segs[-2] in self.enums:
            return "%s.%s" % (segs[-2], last)
        if segs[0] in ("crate", "kernels", "linking", "execute_gpu") and last in self.globals:
            return last
        raise TranslateError("unknown path %s" % full)

    def lit(self, e):
        kind, text = e[1], e[2]
        if kind == "bool":
            return "True" if text == "true" else "False"
        if kind == "str":
            return text.lstrip("b")
        if kind == "chr":
            return repr(text[1:-1])
        t = text.replace("_", "")
        m = re.fullmatch(r"(-?[\d.]+(?:[eE][+-]?\d+)?)(f32|f64|u8|u16|u32|u64|usize|i8|i16|i32|i64|isize)?", t)
        num, suf = m.group(1), m.group(2)
        is_float = suf in ("f32", "f64") or "." in num or "e" in num.lower()
        if is_float:
            return "rt.F32(%r)" % f32_literal(num)
        return str(int(num))

    def is_place(self, e):
        return e[0] in ("path", "field", "index") or (e[0] == "unary" and e[1] == "*") or e[0] == "paren"

    def ref_arg(self, e):
        """Argument passed to a parameter the callee writes through."""
        inner = e
        while inner[0] == "unary" and inner[1] in ("&", "&mut"):
            inner = inner[2]
        if inner[0] == "path" and len(inner[1]) == 1:
            py = self.lookup(inner[1][0])
            if py in self.refs:
                return py
            raise TranslateError("&mut of a local passed to a writing callee: %s" % inner[1][0])
        if inner[0] == "field":
            return "rt.AttrRef(%s, %r)" % (self.expr(inner[1]), inner[2])
        if inner[0] == "index":
            return "rt.IndexRef(%s, %s)" % (self.expr(inner[1]), self.expr(inner[2]))
        raise TranslateError("unsupported reference argument %r" % (inner,))

    def expr(self, e):
        k = e[0]
        if k == "lit":
            return self.lit(e)
        if k == "unit":
            return "None"
        if k == "path":
            return self.path_expr(e[1])
        if k == "paren":
            return "(%s)" % self.expr(e[1])
        if k == "tuple":
            parts = [self.expr(x) for x in e[1]]
            return "(" + ", ".join(parts) + ("," if len(parts) == 1 else "") + ")"
        if k == "array":
            return "[" + ", ".join(self.expr(x) for x in e[1]) + "]"
        if k == "vec_rep":
            return "rt.vec_rep(%s, %s)" % (self.expr(e[1]), self.expr(e[2]))
        if k == "unary":
            op = e[1]
            if op in ("&", "&mut"):
                inner = e[2]
                if op == "&mut" and not self.is_place(inner):
                    return "rt.Cell(%s)" % self.expr(inner)
                return self.expr(inner)
            if op == "*":
                inner = e[2]
                if inner[0] == "path" and len(inner[1]) == 1:
                    py = self.lookup(inner[1][0])
                    if py in self.refs:
                        return "%s.v" % py
                return self.expr(inner)
            if op == "-":
                return "(-%s)" % self.expr(e[2])
            if op == "!":
                return "(not %s)" % self.expr(e[2])
        if k == "binary":
            op, a, b = e[1], e[2], e[3]
            if op == "&&":
                return self.short_circuit("and", a, b)
            if op == "||":
                return self.short_circuit("or", a, b)
            sa, sb = self.expr(a), self.expr(b)
            if op == "/":
                return "rt.div(%s, %s)" % (sa, sb)
            if op == "%":
                return "rt.rem(%s, %s)" % (sa, sb)
            return "(%s %s %s)" % (sa, op, sb)
        if k == "cast":
            ty = TYPE_ALIASES.get(e[2], e[2])
            if ty not in NUM_TYPES:
                raise TranslateError("cast to %s" % ty)
            return "rt.cast(%s, %r)" % (self.expr(e[1]), ty)
        if k == "field":
            base = self.expr(e[1])
            if isinstance(e[2], int):
                return "%s[%d]" % (base, e[2])
            return "%s.%s" % (base, e[2])
        if k == "index":
            base = self.expr(e[1])
            idx = e[2]
            if idx[0] == "array":
                return "%s[%s]" % (base, ", ".join(self.expr(x) for x in idx[1]))
            if idx[0] == "range":
                lo = self.expr(idx[1]) if idx[1] else ""
                hi = self.expr(idx[2]) if idx[2] else ""
                if idx[3] and hi:
                    hi = "(%s) + 1" % hi
                return "%s[%s:%s]" % (base, lo, hi)
            return "%s[%s]" % (base, self.expr(idx))
        if k == "try":
            return self.expr(e[1])
        if k == "mcall":
            recv, name, args = e[1], e[2], e[3]
            r = self.expr(recv)
            if name in IDENTITY_METHODS:
                return r
            a = [self.expr(x) for x in args]
            return "rt.call(%s)" % ", ".join([r, repr(name)] + a)
        if k == "call":
            return self.call_expr(e)
        if k == "range":
            lo = self.expr(e[1]) if e[1] else "0"
            if e[2] is None:
                raise TranslateError("open range outside an index")
            hi = self.expr(e[2])
            if e[3]:
                hi = "(%s) + 1" % hi
            return "range(%s, %s)" % (lo, hi)
        if k == "struct":
            return self.struct_lit(e)
        if k == "closure":
            return self.closure(e)
        if k == "panic":
            return "rt.panic(%r)" % e[1]
        if k == "assert":
            self.emit("assert %s" % self.expr(e[1]))
            return "None"
        if k == "block":
            self.push()
            try:
                for s in e[1]:
                    self.stmt(s)
                return self.expr(e[2]) if e[2] is not None else "None"
            finally:
                self.pop()
        if k in ("if", "match", "loop", "while", "for"):
            t = self.temp()
            self.emit("%s = None" % t)
            self.control(e, t)
            return t
        if k == "assign":
            self.assign(e)
            return "None"
        if k in ("return", "break", "continue"):
            self.control(e, None)
            return "None"
        raise TranslateError("expression %r" % (k,))

    def short_circuit(self, op, a, b):
        mark = len(self.lines)
        sa = self.expr(a)
        mark_b = len(self.lines)
        sb = self.expr(b)
        if len(self.lines) == mark_b:
            return "(%s %s %s)" % (sa, op, sb)
        # b needs statements: evaluate it only when a does not decide
        pre_b = self.lines[mark_b:]
        del self.lines[mark_b:]
        t = self.temp()
        self.emit("%s = %s" % (t, sa))
        self.emit(("if %s:" if op == "and" else "if not %s:") % t)
        self.ind += 1
        for line in pre_b:
            self.lines.append("    " + line)
        self.emit("%s = %s" % (t, sb))
        self.ind -= 1
        del mark
        return t

    def call_expr(self, e):
        fn, args = e[1], e[2]
        if fn[0] == "path":
            segs = fn[1]
            full = "::".join(segs)
            last = segs[-1]
            if full in ("Some", "Ok", "Box::new") and len(args) == 1:
                return self.expr(args[0])
            if full == "Err":
                return "rt.err(%s)" % self.expr(args[0])
            # enum tuple variant of a translated enum
            if len(segs) >= 2 and segs[-2] in self.enums:
                return "%s.%s(%s)" % (segs[-2], last, ", ".join(self.expr(a) for a in args))
            if len(segs) >= 2 and "::".join(segs[:-1]) in ERROR_PREFIXES:
                return "rt.Error(%r, %s)" % (last, ", ".join(self.expr(a) for a in args))
            info = None
            if len(segs) == 1 and self.lookup(last) is None and last in self.fns:
                info = self.fns[last]
            elif len(segs) == 1 and self.lookup(last) is not None and self.lookup(last) in self.fns:
                info = self.fns[self.lookup(last)]
            callee = self.expr(fn)
            out = []
            for i, a in enumerate(args):
                if info is not None and i < len(info.params) and info.params[i] in info.deref:
                    out.append(self.ref_arg(a))
                else:
                    out.append(self.expr(a))
            return "%s(%s)" % (callee, ", ".join(out))
        return "%s(%s)" % (self.expr(fn), ", ".join(self.expr(a) for a in args))

    def struct_lit(self, e):
        segs, fields, base = e[1], e[2], e[3]
        last = segs[-1]
        kw = ", ".join("%s=%s" % (n, self.expr(x)) for n, x in fields)
        head = "::".join(segs[:-1])
        if head in ERROR_PREFIXES:
            return "rt.Error(%r%s)" % (last, (", " + kw) if kw else "")
        if len(segs) >= 2 and segs[-2] in self.enums:
            return "rt.REnum(%r, (), dict(%s))" % (last, kw)
        cls = self.cls if last == "Self" else last
        if base is None or (base[0] == "call" and base[1][0] == "path" and base[1][1][-1] == "default"):
            return "%s(%s)" % (cls, kw)
        return "rt.struct_update(%s, %s%s)" % (cls, self.expr(base), (", " + kw) if kw else "")

    def closure(self, e):
        params, body = e[1], e[2]
        simple = all(p[0] in ("bind", "wild") and (p[0] == "wild" or p[2] is None) for p in params)
        if simple and body[0] != "block":
            mark = len(self.lines)
            saved_tmp = self.tmp
            self.push()
            names = [self.bind(p[1]) if p[0] == "bind" else self.temp("_w") for p in params]
            try:
                s = self.expr(body)
            finally:
                self.pop()
            if len(self.lines) == mark:
                return "(lambda %s: %s)" % (", ".join(names), s)
            del self.lines[mark:]
            self.tmp = saved_tmp
        name = self.temp("_closure")
        self.fn_def(name, [(p, None) for p in params], None, body, closure=True)
        return name

    # --- statements and control flow
    def assign(self, e):
        op, lhs, rhs = e[1], e[2], e[3]
        if lhs[0] == "unary" and lhs[1] == "*" and lhs[2] == ("path", ["self"]):
            self.emit("rt.assign_self(self, %s)" % self.expr(rhs))
            return
        target = self.expr(lhs)
        val = self.expr(rhs)
        if op == "=":
            self.emit("%s = %s" % (target, val))
        elif op == "/=":
            self.emit("%s = rt.div(%s, %s)" % (target, target, val))
        elif op == "%=":
            self.emit("%s = rt.rem(%s, %s)" % (target, target, val))
        else:
            self.emit("%s = %s %s %s" % (target, target, op[:-1], val))

    def stmt(self, s):
        if s[0] == "let":
            pat, init = s[1], s[2]
            if init is None:
                for name in self.pat_names(pat):
                    self.emit("%s = None" % self.bind(name))
                return
            if init[0] == "unary" and init[1] == "&mut" and not self.is_place(init[2]) and pat[0] == "bind":
                val = self.expr(init[2])
                py = self.bind(pat[1])
                self.emit("%s = rt.Cell(%s)" % (py, val))
                self.refs.add(py)
                return
            val = self.expr(init)
            tgt = self.pat_simple_dry(pat)
            if tgt:
                self.emit("%s = %s" % (self.pat_simple(pat), val))
            else:
                t = self.temp()
                self.emit("%s = %s" % (t, val))
                c, binds = self.pat_test(pat, t)
                self.bind_all(binds)
            return
        if s[0] == "letelse":
            t = self.temp()
            self.emit("%s = %s" % (t, self.expr(s[2])))
            c, binds = self.pat_test(s[1], t)
            self.emit("if not (%s):" % c)
            self.ind += 1
            self.tail(s[3], None)
            self.ind -= 1
            self.bind_all(binds)
            return
        if s[0] == "item":
            fn = s[1]
            py = self.bind(fn[1])
            info = FnInfo(py, self.param_names(fn), self.deref_params(fn))
            self.fns[py] = info
            self.fn_def(py, fn[2], fn[3], fn[4], deref=info.deref)
            return
        if s[0] == "expr":
            self.expr_stmt(s[1])
            return
        raise TranslateError("statement %r" % (s[0],))

    def pat_simple_dry(self, p):
        if p[0] == "bind" and p[2] is None:
            return True
        if p[0] == "wild":
            return True
        if p[0] == "ref":
            return self.pat_simple_dry(p[1])
        if p[0] == "ptuple" and all(q[0] != "rest" for q in p[1]):
            return all(self.pat_simple_dry(q) for q in p[1])
        return False

    def pat_names(self, p):
        out = []
        walk(p, lambda n: out.append(n[1]) if n[0] == "bind" else None)
        return out

    def expr_stmt(self, e):
        if e[0] in ("if", "match", "for", "while", "loop", "return", "break", "continue"):
            self.control(e, None)
        elif e[0] == "block":
            self.push()
            for s in e[1]:
                self.stmt(s)
            if e[2] is not None:
                self.expr_stmt(e[2])
            self.pop()
        elif e[0] == "assign":
            self.assign(e)
        else:
            s = self.expr(e)
            if s not in ("None",):
                self.emit(s)

    def tail(self, block, target):
        """Emit a block; its value goes to target (a name, 'return' or None)."""
        self.push()
        try:
            for s in block[1]:
                self.stmt(s)
            t = block[2]
            if t is None:
                if target == "return":
                    self.emit("return None")
                elif target:
                    self.emit("%s = None" % target)
                else:
                    self.emit("pass")
                return
            self.value_to(t, target)
        finally:
            self.pop()

    def value_to(self, e, target):
        if e[0] in ("if", "match", "loop", "block") and target is not None:
            if e[0] == "block":
                self.tail(e, target)
            else:
                self.control(e, target)
            return
        if e[0] in ("return", "break", "continue"):
            self.control(e, None)
            return
        if target is None:
            self.expr_stmt(e)
            self.emit("pass")
        elif target == "return":
            self.emit("return %s" % self.expr(e))
        else:
            self.emit("%s = %s" % (target, self.expr(e)))

    def arm_body(self, body, target):
        if body[0] == "block":
            self.tail(body, target)
        else:
            self.push()
            self.value_to(body, target)
            self.pop()

    def control(self, e, target):
        k = e[0]
        if k == "return":
            if e[1] is None:
                self.emit("return None")
            else:
                v = e[1]
                if v[0] in ("if", "match", "block"):
                    self.value_to(v, "return")
                else:
                    self.emit("return %s" % self.expr(v))
            return
        if k == "break":
            self.emit("break")
            return
        if k == "continue":
            self.emit("continue")
            return
        if k == "if":
            cond, then, els = e[1], e[2], e[3]
            if cond[0] == "let":
                s = self.temp("_s")
                self.emit("%s = %s" % (s, self.expr(cond[2])))
                c, binds = self.pat_test(cond[1], s)
                self.emit("if %s:" % c)
                self.ind += 1
                self.push()
                self.bind_all(binds)
                self.tail(then, target)
                self.pop()
                self.ind -= 1
            else:
                c = self.expr(cond)
                self.emit("if %s:" % c)
                self.ind += 1
                self.tail(then, target)
                self.ind -= 1
            if els is not None:
                self.emit("else:")
                self.ind += 1
                if els[0] == "if":
                    self.control(els, target)
                else:
                    self.tail(els, target)
                self.ind -= 1
            elif target not in (None, "return"):
                self.emit("else:")
                self.emit("    %s = None" % target)
            return
        if k == "match":
            s = self.temp("_s")
            self.emit("%s = %s" % (s, self.expr(e[1])))
            arms = e[2]
            if any(g is not None for _, g, _ in arms):
                done = self.temp("_m")
                self.emit("%s = False" % done)
                for pat, guard, body in arms:
                    c, binds = self.pat_test(pat, s)
                    self.emit("if not %s and (%s):" % (done, c))
                    self.ind += 1
                    self.push()
                    self.bind_all(binds)
                    if guard is not None:
                        self.emit("if %s:" % self.expr(guard))
                        self.ind += 1
                    self.emit("%s = True" % done)
                    self.arm_body(body, target)
                    if guard is not None:
                        self.ind -= 1
                    self.pop()
                    self.ind -= 1
                self.emit("if not %s:" % done)
                self.emit("    rt.panic('non-exhaustive match')")
                return
            first = True
            exhaustive = False
            for pat, guard, body in arms:
                c, binds = self.pat_test(pat, s)
                if c == "False":
                    continue   # an arm that only matches Err values never runs
                if c == "True":
                    self.emit("else:" if not first else "if True:")
                    exhaustive = True
                else:
                    self.emit(("if %s:" if first else "elif %s:") % c)
                self.ind += 1
                self.push()
                self.bind_all(binds)
                self.arm_body(body, target)
                self.pop()
                self.ind -= 1
                first = False
                if exhaustive:
                    break
            if not exhaustive:
                self.emit("else:")
                self.emit("    rt.panic('non-exhaustive match')")
            return
        if k == "for":
            pat, it, body = e[1], e[2], e[3]
            self.for_loop(pat, it, body)
            return
        if k == "while":
            cond, body = e[1], e[2]
            if cond[0] == "let":
                self.emit("while True:")
                self.ind += 1
                s = self.temp("_s")
                self.emit("%s = %s" % (s, self.expr(cond[2])))
                c, binds = self.pat_test(cond[1], s)
                self.emit("if not (%s):" % c)
                self.emit("    break")
                self.push()
                self.bind_all(binds)
                self.tail(body, None)
                self.pop()
                self.ind -= 1
                return
            mark = len(self.lines)
            c = self.expr(cond)
            if len(self.lines) == mark:
                self.emit("while %s:" % c)
                self.ind += 1
                self.tail(body, None)
                self.ind -= 1
                return
            del self.lines[mark:]
            self.emit("while True:")
            self.ind += 1
            c = self.expr(cond)
            self.emit("if not %s:" % c)
            self.emit("    break")
            self.tail(body, None)
            self.ind -= 1
            return
        if k == "loop":
            self.emit("while True:")
            self.ind += 1
            self.tail(e[1], None)
            self.ind -= 1
            return
        if k == "block":
            self.tail(e, target)
            return
        raise TranslateError("control %r" % (k,))

    def derefs_of(self, body, name):
        found = []

        def f(n):
            if n[0] == "unary" and n[1] == "*" and n[2] == ("path", [name]):
                found.append(n)
        walk(body, f)
        return bool(found)

    def for_loop(self, pat, it, body):
        inner = it
        while inner[0] == "unary" and inner[1] in ("&", "&mut"):
            inner = inner[2]
        # `for v in x.iter_mut() { *v = ... }`: assign through the element places
        if inner[0] == "mcall" and inner[2] == "iter_mut" and pat[0] == "bind" and self.derefs_of(body, pat[1]):
            lst = self.temp("_l")
            i = self.temp("_i")
            self.emit("%s = %s" % (lst, self.expr(inner[1])))
            self.emit("for %s in range(len(%s)):" % (i, lst))
            self.ind += 1
            self.push()
            py = self.bind(pat[1])
            self.alias[py] = "%s[%s]" % (lst, i)
            self.tail(body, None)
            self.alias.pop(py, None)
            self.pop()
            self.ind -= 1
            return
        if inner[0] == "range" and inner[1] is not None and inner[2] is not None:
            src = self.expr(inner)
        else:
            src = "rt.iterate(%s)" % self.expr(inner)
        self.push()
        tgt = self.pat_simple(pat) if self.pat_simple_dry(pat) else None
        if tgt:
            self.emit("for %s in %s:" % (tgt, src))
            self.ind += 1
        else:
            v = self.temp("_v")
            self.emit("for %s in %s:" % (v, src))
            self.ind += 1
            c, binds = self.pat_test(pat, v)
            self.bind_all(binds)
        self.tail(body, None)
        self.ind -= 1
        self.pop()

    # --- functions
    def param_names(self, fn):
        return [p[0][1] if p[0][0] == "bind" else None for p in fn[2]]

    def deref_params(self, fn):
        names = set(n for n in self.param_names(fn) if n)
        out = set()

        def f(n):
            if n[0] == "unary" and n[1] == "*" and n[2][0] == "path" and len(n[2][1]) == 1 \
                    and n[2][1][0] in names:
                out.add(n[2][1][0])
        walk(fn[4], f)
        # derefs of Copy elements (`*dest.0`) are plain reads; only names count
        return out

    def fn_def(self, name, params, self_kind, body, closure=False, deref=None):
        assigned_outer = set()
        if closure:
            lets = set()

            def f(n):
                if n[0] == "let":
                    lets.update(self.pat_names(n[1]))
                if n[0] == "assign" and n[2][0] == "path" and len(n[2][1]) == 1:
                    tgt = n[2][1][0]
                    if tgt not in lets and self.lookup(tgt) is not None:
                        assigned_outer.add(self.lookup(tgt))
            walk(body, f)
        saved_scopes = self.scopes
        saved_refs, saved_alias = set(self.refs), dict(self.alias)
        if not closure:
            # a nested fn sees the fn items of the blocks around it, not their locals
            items = {}
            for sc in self.scopes:
                for rn, py in sc.items():
                    if py in self.fns:
                        items[rn] = py
            self.scopes = [items, {}]
            self.refs = set()
            self.alias = {}
        else:
            self.scopes = self.scopes + [{}]
        pnames = []
        destructure = []
        for i, (p, _ty) in enumerate(params):
            if p[0] == "bind" and p[2] is None:
                pnames.append(self.bind(p[1]))
            elif p[0] == "wild":
                pnames.append(self.temp("_w"))
            else:
                t = self.temp("_p")
                pnames.append(t)
                destructure.append((p, t))
        if self_kind:
            pnames.insert(0, "self")
        self.emit("def %s(%s):" % (name, ", ".join(pnames)))
        self.ind += 1
        if assigned_outer:
            self.emit("nonlocal " + ", ".join(sorted(assigned_outer)))
        if deref:
            for n in deref:
                py = self.lookup(n)
                if py:
                    self.refs.add(py)
        for p, t in destructure:
            if self.pat_simple_dry(p):
                self.emit("%s = %s" % (self.pat_simple(p), t))
            else:
                c, binds = self.pat_test(p, t)
                self.bind_all(binds)
        if body[0] == "block":
            self.tail(body, "return")
        else:
            self.emit("return %s" % self.expr(body))
        self.ind -= 1
        self.scopes = saved_scopes
        self.refs, self.alias = saved_refs, saved_alias

    def top_fn(self, fn, pyname=None):
        info = FnInfo(fn[1], self.param_names(fn), self.deref_params(fn))
        self.used = set()
        self.tmp = 0
        self.fn_def(pyname or fn[1], fn[2], fn[3], fn[4], deref=info.deref)


# ------------------------------------------------------------------ driver
def field_default(ty):
    base = ty.lstrip("&").split("::")[-1]
    base = TYPE_ALIASES.get(base, base)
    if base in ("f32", "f64"):
        return "rt.F32(0.0)"
    if base in NUM_TYPES and base != "bool":
        return "0"
    if base == "bool":
        return "False"
    if base in ("Vec",) or ty.startswith("["):
        return "list"
    return "None"


def extract_fragment(src, first, last, head, tail):
    lines = src.split("\n")
    start = next(i for i, l in enumerate(lines) if re.search(first, l))
    end = next(i for i in range(start + 1, len(lines)) if re.search(last, lines[i]))
    return head + "\n" + "\n".join(lines[start:end + 1]) + "\n" + tail + "\n", start + 1, end + 1


def translate(ref_root):
    files = {}
    for f in sorted(set(x[0] for x in ITEMS) | set(x[0] for x in FRAGMENTS)):
        with open(os.path.join(ref_root, f)) as fh:
            files[f] = fh.read()
    def wanted_in(f):
        names = set((k, n) for ff, k, n in ITEMS if ff == f)
        return lambda kind, name: (kind, name) in names or (kind == "fn" and ("fn", name) in names)
    parsed = {f: Parser(lex(s), wanted_in(f)).parse_items() for f, s in files.items()}
    wanted = []
    for f, kind, name in ITEMS:
        found = [it for it in parsed[f] if it[0] == kind and it[1] == name]
        if not found:
            raise TranslateError("%s %s not found in %s" % (kind, name, f))
        wanted.extend((f, it) for it in found)
    frag_fns = []
    for f, first, last, head, tail in FRAGMENTS:
        text, l0, l1 = extract_fragment(files[f], first, last, head, tail)
        items = Parser(lex(text)).parse_items()
        frag_fns.append(((f, l0, l1), items[0]))

    em = Emitter()
    for _f, it in wanted:
        if it[0] in ("struct", "fn"):
            em.globals.add(it[1])
        if it[0] == "struct":
            em.structs[it[1]] = it[2]
        if it[0] == "enum":
            em.globals.add(it[1])
            em.enums[it[1]] = it[2]
        if it[0] == "fn":
            em.fns[it[1]] = FnInfo(it[1], em.param_names(it), em.deref_params(it))
    for _src, fn in frag_fns:
        em.globals.add(fn[1])
        em.fns[fn[1]] = FnInfo(fn[1], em.param_names(fn), em.deref_params(fn))

    out = ['"""Generated by oracle/rust2py.py from the reference checkout; do not edit."""',
           "import rust_rt as rt", "", ""]
    em.lines = out
    # structs and enums first (impls attach methods to them)
    for f, it in wanted:
        if it[0] == "struct":
            em.emit("class %s(rt.Struct):" % it[1])
            em.emit("    # %s" % f)
            em.emit("    _fields = (%s)" % "".join("(%r, %s), " % (n, field_default(t)) for n, t in it[2]))
            em.emit("")
            em.emit("")
        elif it[0] == "enum":
            em.emit("class %s(rt.REnum):" % it[1])
            em.emit("    # %s" % f)
            em.emit("    pass")
            em.emit("")
            em.emit("")
            for vname, vkind in it[2]:
                if vkind == "unit":
                    em.emit("%s.%s = %s(%r)" % (it[1], vname, it[1], vname))
                else:
                    em.emit("%s.%s = staticmethod(lambda *a: %s(%r, a))" % (it[1], vname, it[1], vname))
            em.emit("")
    for f, it in wanted:
        if it[0] == "fn":
            em.emit("# %s: fn %s" % (f, it[1]))
            em.top_fn(it)
            em.emit("")
            em.emit("")
        elif it[0] == "impl":
            target, trait, fns = it[1], it[2], it[3]
            holder = target if target in em.structs or target in em.enums else "rt." + target
            em.cls = holder
            for fn in fns:
                em.emit("# %s: impl %s%s :: %s" % (f, (trait + " for ") if trait else "", target, fn[1]))
                mangled = "_m_%s_%s" % (target, fn[1])
                em.top_fn(fn, mangled)
                em.emit("%s.%s = %s" % (holder, fn[1], mangled) if fn[3] else
                        "%s.%s = staticmethod(%s)" % (holder, fn[1], mangled))
                if trait and trait.split("::")[-1] == "Index" and fn[1] == "index":
                    em.emit("%s.__getitem__ = %s" % (holder, mangled))
                if trait and trait.split("::")[-1] == "Iterator" and fn[1] == "next":
                    em.emit("%s.__iter__ = lambda self: rt.from_next(self)" % holder)
                em.emit("")
            em.cls = None
    for (f, l0, l1), fn in frag_fns:
        em.emit("# %s:%d-%d, wrapped in fn %s" % (f, l0, l1, fn[1]))
        em.top_fn(fn)
        em.emit("")
        em.emit("")
    return "\n".join(out) + "\n"


def main():
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    ref_root, out_dir = sys.argv[1], sys.argv[2]
    os.makedirs(out_dir, exist_ok=True)
    code = translate(ref_root)
    compile(code, "rust_ref.py", "exec")
    with open(os.path.join(out_dir, "rust_ref.py"), "w") as f:
        f.write(code)
    print("wrote %s" % os.path.join(out_dir, "rust_ref.py"))


if __name__ == "__main__":
    main()
