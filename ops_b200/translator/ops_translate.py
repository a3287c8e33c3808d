"""Source-to-source translator: OPS application -> B200 (sm_100a) build.

Plays the role of the reference's code generators
(ops_translator/ops-translator/ with the templates in
ops_translator/resources/templates/cpp/cuda/loop_host.cpp.j2, and the legacy
ops_translator_legacy/c/ops_gen_mpi_cuda.py): every ``ops_par_loop`` call site
is rewritten into a call of a generated host stub, and every distinct loop gets
one hand-written-style CUDA kernel.  The parser is this project's own (a small
comment/string-aware scanner; libclang is not needed).

Output for an application made of sources S1.cpp ... Sn.cpp:
  * ``S_ops.cpp`` per source: the source with ``ops_seq_v2.h`` replaced by the
    backend headers plus stub prototypes, and ``ops_par_loop(k, ...)`` replaced
    by ``ops_par_loop_<k>(...)``;
  * ``<app>_kernels.cu``: all user kernels (copied verbatim as __device__
    functions), every ``ops_decl_const`` as a __constant__ symbol, one
    __global__ kernel and one host stub per loop, and the constant copier.

Kernel shape (per loop): one thread per grid point; x on threadIdx.x so that
every dat access of a warp is one contiguous run along x; CTA shape from the
runtime (OPS_BLOCK_SIZE_X/Y/Z, default 32x4x1); ops_arg_gbl(READ) values are
passed by value inside the kernel parameters (copied at call time, the
reference's lazy semantics, ops_lazy.cpp:1433-1437); reductions go through
the warp-shuffle / last-CTA combine of include/ops_b200_kernel.h.
"""

from __future__ import annotations

import argparse
import os
import re
import sys
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

from .divrewrite import macro_table, rewrite_divisions

# --------------------------------------------------------------------------
# scanning helpers
# --------------------------------------------------------------------------


def mask_comments_strings(src: str, keep_strings: bool = False) -> str:
    """Return src with comments (and, unless keep_strings, string/char
    literal contents) replaced by spaces; offsets and newlines preserved."""
    out = list(src)
    i, n = 0, len(src)
    while i < n:
        c = src[i]
        if c == "/" and i + 1 < n and src[i + 1] == "/":
            j = src.find("\n", i)
            j = n if j < 0 else j
            for k in range(i, j):
                out[k] = " "
            i = j
        elif c == "/" and i + 1 < n and src[i + 1] == "*":
            j = src.find("*/", i + 2)
            j = n if j < 0 else j + 2
            for k in range(i, j):
                if src[k] != "\n":
                    out[k] = " "
            i = j
        elif c in "\"'":
            q = c
            j = i + 1
            while j < n and src[j] != q:
                if src[j] == "\\":
                    j += 1
                j += 1
            if not keep_strings:
                for k in range(i + 1, min(j, n)):
                    if src[k] != "\n":
                        out[k] = " "
            i = j + 1
        else:
            i += 1
    return "".join(out)


def match_paren(masked: str, open_idx: int) -> int:
    """Index of the bracket closing the one at open_idx (in masked text)."""
    pairs = {"(": ")", "{": "}", "[": "]"}
    opener = masked[open_idx]
    closer = pairs[opener]
    depth = 0
    for i in range(open_idx, len(masked)):
        ch = masked[i]
        if ch == opener:
            depth += 1
        elif ch == closer:
            depth -= 1
            if depth == 0:
                return i
    raise ValueError("unbalanced bracket at offset %d" % open_idx)


def split_top(text: str, masked: str) -> List[str]:
    """Split text at top-level commas (masked guides the nesting)."""
    parts, depth, start = [], 0, 0
    for i, ch in enumerate(masked):
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        elif ch == "," and depth == 0:
            parts.append(text[start:i].strip())
            start = i + 1
    tail = text[start:].strip()
    if tail or parts:
        parts.append(tail)
    return parts


def find_calls(src: str, name: str) -> List[Tuple[int, int, List[str]]]:
    """All calls `name(...)`: (start, end_exclusive, args)."""
    masked = mask_comments_strings(src)
    res = []
    for m in re.finditer(r"(?<![\w.>])" + re.escape(name) + r"\s*\(", masked):
        op = m.end() - 1
        cl = match_paren(masked, op)
        args = split_top(src[op + 1:cl], masked[op + 1:cl])
        res.append((m.start(), cl + 1, args))
    return res


def unquote(s: str) -> str:
    s = s.strip()
    if len(s) >= 2 and s[0] == '"' and s[-1] == '"':
        return s[1:-1]
    return s


# --------------------------------------------------------------------------
# model
# --------------------------------------------------------------------------


@dataclass
class LoopArg:
    kind: str  # dat | gbl | reduce | idx
    ctype: str = ""  # element type string
    dim: str = "1"  # dimension expression
    acc: str = "OPS_READ"
    opt: bool = False
    stencil: str = ""  # the stencil expression of a dat argument
    prolong: bool = False  # the stencil was declared by ops_decl_prolong_stencil

    def key(self) -> Tuple:
        return (self.kind, self.ctype, self.dim if self.kind != "dat" else
                ("1" if self.dim.strip() == "1" else "n"), self.acc, self.opt, self.prolong)


@dataclass
class KernelParam:
    text: str
    base_type: str  # e.g. double
    is_acc: bool
    is_const: bool
    name: str


@dataclass
class KernelDef:
    name: str
    params: List[KernelParam]
    text: str  # full definition text
    header: str  # file it came from


@dataclass
class Loop:
    kernel: str
    ndim: int
    args: List[LoopArg]
    stub: str = ""
    sources: List[str] = field(default_factory=list)

    def key(self) -> Tuple:
        return (self.kernel, self.ndim, tuple(a.key() for a in self.args))


@dataclass
class ConstDecl:
    name: str
    dim: str
    ctype: str


ACCESS = {"OPS_READ", "OPS_WRITE", "OPS_RW", "OPS_INC", "OPS_MIN", "OPS_MAX"}
OB2_MAX_ACC_MACROS = 48  # OPS_ACCn / OPS_ACC_MDn macros given a host meaning


def parse_arg(text: str, where: str) -> LoopArg:
    masked = mask_comments_strings(text)
    m = re.match(r"\s*(ops_arg_\w+)\s*\(", masked)
    if not m:
        raise SystemExit("%s: cannot parse ops_par_loop argument: %s" % (where, text))
    fn = m.group(1)
    op = m.end() - 1
    cl = match_paren(masked, op)
    inner = split_top(text[op + 1:cl], masked[op + 1:cl])
    if fn == "ops_arg_dat":
        if len(inner) != 5:
            raise SystemExit("%s: ops_arg_dat needs 5 arguments: %s" % (where, text))
        return LoopArg("dat", unquote(inner[3]), inner[1], inner[4].strip(),
                       stencil=inner[2].strip())
    if fn == "ops_arg_dat_opt":
        if len(inner) != 6:
            raise SystemExit("%s: ops_arg_dat_opt needs 6 arguments: %s" % (where, text))
        return LoopArg("dat", unquote(inner[3]), inner[1], inner[4].strip(), opt=True,
                       stencil=inner[2].strip())
    if fn == "ops_arg_gbl":
        if len(inner) != 4:
            raise SystemExit("%s: ops_arg_gbl needs 4 arguments: %s" % (where, text))
        acc = inner[3].strip()
        if acc != "OPS_READ":
            raise SystemExit("%s: ops_arg_gbl supports OPS_READ only; use ops_arg_reduce" % where)
        return LoopArg("gbl", unquote(inner[2]), inner[1], acc)
    if fn == "ops_arg_reduce":
        if len(inner) != 4:
            raise SystemExit("%s: ops_arg_reduce needs 4 arguments: %s" % (where, text))
        acc = inner[3].strip()
        if acc not in ("OPS_INC", "OPS_MIN", "OPS_MAX"):
            raise SystemExit("%s: ops_arg_reduce access must be INC/MIN/MAX" % where)
        return LoopArg("reduce", unquote(inner[2]), inner[1], acc)
    if fn == "ops_arg_idx":
        return LoopArg("idx", "int", "3", "OPS_READ")
    raise SystemExit("%s: unsupported argument kind %s" % (where, fn))


def parse_params(ptext: str) -> List[KernelParam]:
    masked = mask_comments_strings(ptext)
    out = []
    for p in split_top(ptext, masked):
        if not p or p == "void":
            continue
        t = re.sub(r"\s+", " ", p.strip())
        m = re.match(r"^(const\s+)?ACC\s*<\s*([\w\s:]+?)\s*>\s*&?\s*(\w+)$", t)
        if m:
            out.append(KernelParam(p, m.group(2).strip(), True, bool(m.group(1)), m.group(3)))
            continue
        m = re.match(r"^(const\s+)?([\w\s:]+?)\s*(const\s*)?\*\s*(?:__restrict__\s*|restrict\s*)?(\w+)$", t)
        if m:
            out.append(KernelParam(p, m.group(2).strip(), False,
                                   bool(m.group(1) or m.group(3)), m.group(4)))
            continue
        raise SystemExit("unsupported kernel parameter form: '%s'" % p)
    return out


FUNC_RE = re.compile(
    r"((?:(?:static|inline|__forceinline__|__host__|__device__|OPS_FUN_PREFIX|constexpr)\s+)*)"
    r"([\w:<>\s\*&]+?)\s*\b(\w+)\s*\(([^{};]*)\)\s*(?:const\s*)?$", re.S)


def top_level_functions(text: str, header: str) -> List[KernelDef]:
    """Top-level function definitions of a header (name, params, full text)."""
    masked = mask_comments_strings(text)
    # drop preprocessor lines from consideration (keep offsets)
    lines = masked.split("\n")
    pos = 0
    masked_l = list(masked)
    for ln in lines:
        if ln.lstrip().startswith("#"):
            for k in range(pos, pos + len(ln)):
                masked_l[k] = " "
        pos += len(ln) + 1
    masked = "".join(masked_l)
    res = []
    depth = 0
    i = 0
    last_stmt_end = 0
    n = len(masked)
    while i < n:
        ch = masked[i]
        if ch == "{" and depth == 0:
            head = masked[last_stmt_end:i]
            close = match_paren(masked, i)
            m = FUNC_RE.search(head.strip())
            hs = head.strip()
            if m and not re.match(r"^(struct|class|union|enum|namespace|extern)\b", hs) \
                    and m.group(3) not in ("if", "for", "while", "switch"):
                start = last_stmt_end + (len(head) - len(head.lstrip()))
                full = text[start:close + 1]
                seg = masked[last_stmt_end:i]
                try:
                    params = parse_params(seg[seg.index("(", seg.find(m.group(3))) + 1:
                                              seg.rindex(")")])
                except SystemExit:
                    params = None
                res.append((m.group(3), params, full))
            i = close + 1
            last_stmt_end = i
            continue
        if ch == ";" and depth == 0:
            last_stmt_end = i + 1
        i += 1
    return [KernelDef(nm, prm, full, header) for nm, prm, full in res]


# --------------------------------------------------------------------------
# translator
# --------------------------------------------------------------------------


class Translator:
    def __init__(self, sources: List[str], include_dirs: List[str], app: str, outdir: str):
        self.sources = sources
        self.include_dirs = include_dirs
        self.app = app
        self.outdir = outdir
        self.loops: Dict[Tuple, Loop] = {}
        self.call_sites: Dict[str, List[Tuple[int, int, str]]] = {}
        self.consts: Dict[str, ConstDecl] = {}
        self.kernels: Dict[str, KernelDef] = {}
        self.helpers: Dict[str, KernelDef] = {}
        self.headers: List[str] = []
        self.header_includes: List[str] = []
        self.ndim = 0
        # code-generation knobs (build-time environment): points per thread
        # along y for non-reduction loops, and the minimum resident CTAs per
        # SM given to __launch_bounds__ (caps registers per thread; default 4,
        # measured fastest on the CloverLeaf step: more resident warps
        # outweigh the few small register spills it causes)
        self.py_forced = "OPS_B200_PY" in os.environ
        self.py = max(1, int(os.environ.get("OPS_B200_PY", "1")))
        # strided rows per trip of a reduction kernel's row loop (at least)
        self.rpy = max(1, int(os.environ.get("OPS_B200_RPY", "1")))
        self.light_max = int(os.environ.get("OPS_B200_LIGHT", "4"))
        # OPS_B200_CHECK=1: OPS_ACCn accesses are checked against their dat's
        # allocation; an access outside it prints its kernel, argument, point
        # and offset (device printf) and is redirected to the dat's first
        # element instead of being made
        self.check = os.environ.get("OPS_B200_CHECK", "0") == "1"
        self.minb = max(0, int(os.environ.get("OPS_B200_MINB", "4")))
        # OPS_B200_DDIV=0: user kernels keep their `/` operators; otherwise
        # every division the scanner can group safely becomes ob2::div
        # (include/ops_b200_kernel.h: correctly rounded, the same bits)
        self.ddiv = os.environ.get("OPS_B200_DDIV", "1") != "0"
        self.div_counts = [0, 0]

    # -- discovery ---------------------------------------------------------
    def resolve_include(self, name: str, from_dir: str) -> Optional[str]:
        for d in [from_dir] + self.include_dirs:
            p = os.path.join(d, name)
            if os.path.isfile(p):
                return os.path.abspath(p)
        return None

    def quoted_includes(self, path: str) -> List[str]:
        try:
            src = mask_comments_strings(open(path).read(), keep_strings=True)
        except OSError:
            return []
        res = []
        for m in re.finditer(r'^\s*#\s*include\s*"([^"]+)"', src, re.M):
            inc = m.group(1)
            if inc.startswith("ops_") or not inc.endswith(".h"):
                continue
            p = self.resolve_include(inc, os.path.dirname(path))
            if p:
                res.append(p)
        return res

    def scan_headers(self, path: str, seen: set) -> None:
        for p in self.quoted_includes(path):
            if p not in seen:
                seen.add(p)
                self.headers.append(p)
                self.scan_headers(p, seen)

    @staticmethod
    def is_kernel_header(path: str) -> bool:
        b = os.path.basename(path)
        return b.endswith("kernel.h") or b.endswith("kernels.h")

    def cu_includes(self) -> List[str]:
        """Headers the device code needs: user_types.h (OPS convention for
        types shared with kernels) and whatever the kernel headers include."""
        out: List[str] = []
        dirs = {os.path.dirname(s) for s in self.sources} | set(self.include_dirs)
        for d in sorted(dirs):
            p = os.path.join(d, "user_types.h")
            if os.path.isfile(p) and os.path.abspath(p) not in out:
                out.append(os.path.abspath(p))

        def walk(h: str, seen: set) -> None:
            for p in self.quoted_includes(h):
                if p in seen or self.is_kernel_header(p):
                    continue
                seen.add(p)
                walk(p, seen)
                if p not in out:
                    out.append(p)
        seen: set = set()
        for h in self.headers:
            if self.is_kernel_header(h):
                walk(h, seen)
        return out

    def run(self) -> None:
        seen: set = set()
        for s in self.sources:
            self.scan_headers(s, seen)
        for h in self.headers:
            text = open(h).read()
            for kd in top_level_functions(text, h):
                if kd.params is not None and kd.name not in self.kernels:
                    self.kernels[kd.name] = kd
                self.helpers.setdefault(kd.name, kd)
        # multigrid prolong stencils (ops_lib_core.cpp:785-831): a dat argument
        # whose stencil variable was declared by ops_decl_prolong_stencil reads
        # its dat at the loop index divided by the multigrid stride, which the
        # generated code computes (restrict stencils scale the index, which
        # the runtime folds into the argument's steps)
        self.prolong_names = set()
        for s in self.sources:
            for m in re.finditer(r"\b(\w+)\s*=\s*ops_decl_prolong_stencil\s*\(",
                                 mask_comments_strings(open(s).read())):
                self.prolong_names.add(m.group(1))
        for s in self.sources:
            src = open(s).read()
            m = re.search(r"#\s*define\s+OPS_(\d)D\b", src)
            if m:
                self.ndim = max(self.ndim, int(m.group(1)))
            self.parse_source(s, src)
        if self.ndim == 0:
            self.ndim = max([l.ndim for l in self.loops.values()] + [2])
        self.assign_stub_names()
        os.makedirs(self.outdir, exist_ok=True)
        for s in self.sources:
            self.write_source(s)
        self.write_kernels()

    def parse_source(self, path: str, src: str) -> None:
        where = os.path.basename(path)
        sites = []
        for start, end, args in find_calls(src, "ops_par_loop"):
            if len(args) < 5:
                raise SystemExit("%s: ops_par_loop with fewer than 5 arguments" % where)
            kname = args[0].strip()
            try:
                ndim = int(args[3].strip())
            except ValueError:
                raise SystemExit("%s: ops_par_loop dim must be a literal: %s" % (where, args[3]))
            largs = [parse_arg(a, where) for a in args[5:]]
            for a in largs:
                if a.kind == "dat" and a.stencil in self.prolong_names:
                    a.prolong = True
            loop = Loop(kname, ndim, largs)
            k = loop.key()
            if k not in self.loops:
                self.loops[k] = loop
            self.loops[k].sources.append(where)
            sites.append((start, end, k, args))
        self.call_sites[path] = sites
        # free calls, and the member calls of the C++ object API
        # (instance->decl_const(...), instance->update_const(...))
        member = []
        masked = mask_comments_strings(src)
        for m in re.finditer(r"(?:->|\.)\s*(?:decl_const|update_const)\s*\(", masked):
            op = m.end() - 1
            cl = match_paren(masked, op)
            member.append((m.start(), cl + 1, split_top(src[op + 1:cl], masked[op + 1:cl])))
        for fn in ("ops_decl_const", "ops_decl_const2", "ops_update_const", None):
            for _, _, args in (find_calls(src, fn) if fn else member):
                if len(args) != 4:
                    continue
                name = unquote(args[0])
                ctype = unquote(args[2]).split(":")[0].strip()
                if name not in self.consts:
                    self.consts[name] = ConstDecl(name, args[1].strip(), ctype)

    def assign_stub_names(self) -> None:
        used: Dict[str, int] = {}
        for k, loop in self.loops.items():
            n = used.get(loop.kernel, 0)
            used[loop.kernel] = n + 1
            loop.stub = "ops_par_loop_%s" % loop.kernel + ("" if n == 0 else "_v%d" % n)

    # -- source rewrite ------------------------------------------------------
    def stub_proto(self, loop: Loop) -> str:
        args = ", ".join("ops_arg" for _ in loop.args)
        return "void %s(char const *, ops_block, int, int *%s);" % (
            loop.stub, (", " + args) if args else "")

    def write_source(self, path: str) -> None:
        src = open(path).read()
        sites = self.call_sites.get(path, [])
        out = []
        last = 0
        for start, end, k, args in sites:
            loop = self.loops[k]
            out.append(src[last:start])
            out.append("%s(%s)" % (loop.stub, ", ".join(args[1:])))
            last = end
        out.append(src[last:])
        body = "".join(out)
        protos = "\n".join(self.stub_proto(l) for l in self.loops.values())
        # host code never runs kernel bodies (the stubs launch the device
        # copies), but it may include kernel headers written with OPS_ACCn
        # index macros: give them an empty host meaning
        acc_macros = "".join("#ifndef OPS_ACC%d\n#define OPS_ACC%d(...) 0\n#endif\n"
                             "#ifndef OPS_ACC_MD%d\n#define OPS_ACC_MD%d(...) 0\n#endif\n" %
                             (i, i, i, i) for i in range(OB2_MAX_ACC_MACROS))
        hdr = ('#include "ops_lib_core.h"\n#include "ops_tridiag.h"\n%s'
               "/* generated par_loop stubs (B200 backend) */\n%s\n" % (acc_macros, protos))
        body, nsub = re.subn(r'^\s*#\s*include\s*[<"]ops_seq(_v2)?\.h[>"].*$', hdr.rstrip("\n"),
                             body, count=1, flags=re.M)
        if nsub == 0:
            body = hdr + body
        base = os.path.splitext(os.path.basename(path))[0]
        with open(os.path.join(self.outdir, base + "_ops.cpp"), "w") as f:
            f.write("/* generated from %s by the OPS B200 translator */\n" % os.path.basename(path))
            f.write('#line 1 "%s"\n' % os.path.abspath(path))
            f.write(body)

    # -- kernels file --------------------------------------------------------
    def const_decl(self, c: ConstDecl) -> str:
        d = c.dim.strip()
        if d == "1":
            return "__constant__ %s %s;" % (c.ctype, c.name)
        if re.fullmatch(r"\d+", d):
            return "__constant__ %s %s[%s];" % (c.ctype, c.name, d)
        # run-time length: fixed-capacity symbol, checked at copy time
        return "__constant__ %s %s[OB2_CONST_CAP(%s)];" % (c.ctype, c.name, c.ctype)

    def write_kernels(self) -> None:
        L: List[str] = []
        w = L.append
        w("/* generated by the OPS B200 translator: kernels of application '%s' */" % self.app)
        w("#define OPS_%dD" % self.ndim)
        w("#ifndef OPS_FUN_PREFIX")
        w("#define OPS_FUN_PREFIX __host__ __device__")
        w("#endif")
        w('#include "ops_lib_core.h"')
        w('#include "ops_b200_loop.h"')
        w('#include "ops_b200_kernel.h"')
        w("#include <cuda_runtime.h>")
        w("#include <algorithm>")
        # user headers that kernel headers depend on (types, macros)
        for h in self.cu_includes():
            w('#include "%s"' % h)
        w("#define OB2_CONST_CAP(T) ((4096 + sizeof(T) - 1) / sizeof(T))")
        w("namespace ob2_%s {" % re.sub(r"\W", "_", self.app))
        # the application's fused launcher (defined after all loops)
        w("static int ob2f_launch(int n, const int *ids, const void *const *prm,"
          " const size_t *psz, const unsigned *grids, const unsigned *block, int idx32,"
          " void *st);")
        self.fuse_items = []
        for c in self.consts.values():
            w(self.const_decl(c))
        # all functions of the kernel headers, as device functions
        # kernels written with pointers and OPS_ACCn(x, y, z) index macros
        # (the reference's original API) take their dat arguments as
        # pointers to the point plus, per such argument, the element strides
        # along x, y, z and between components
        legacy = {}
        for loop in self.loops.values():
            kd = self.kernels.get(loop.kernel)
            if kd is None or kd.params is None:
                continue
            idx = [i for i, (a, p) in enumerate(zip(loop.args, kd.params))
                   if a.kind == "dat" and not p.is_acc]
            if idx:
                legacy[loop.kernel] = (loop.ndim, idx)

        macros = None
        if self.ddiv:
            texts = []
            for f in list(self.sources) + list(self.headers) + [
                    os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(
                        os.path.abspath(__file__)))), "include", "ops_lib_core.h")]:
                try:
                    texts.append(open(f).read())
                except OSError:
                    pass
            macros = macro_table(texts)

        def divisions(text: str) -> str:
            """the function with its body's divisions rewritten"""
            if macros is None:
                return text
            masked = mask_comments_strings(text)
            lb = masked.find("{")
            if lb < 0:
                return text
            body, done, kept = rewrite_divisions(text[lb:], mask_comments_strings, macros)
            self.div_counts[0] += done
            self.div_counts[1] += kept
            return text[:lb] + body

        def emit_fn(kd):
            text = divisions(re.sub(r"^\s*(static\s+|inline\s+)*", "", kd.text))
            if kd.name not in legacy:
                if re.search(r"\bOPS_ACC(_MD)?\d+\s*\(", mask_comments_strings(text)):
                    return  # an OPS_ACCn kernel no loop of this program calls
                w("static __device__ __forceinline__ " + text)
                return
            nd, idx = legacy[kd.name]
            coords = ["x", "y", "z"][:max(1, min(3, nd))]
            for i in idx:
                expr = " + ".join("(%s) * ob2_s%s%d" % (c, c, i) for c in coords)
                if self.check:
                    w("#define OPS_ACC%d(%s) ob2_chk(%s, ob2_lo%d, ob2_hi%d, \"%s\", %d)" %
                      (i, ", ".join(coords), expr, i, i, kd.name, i))
                    w("#define OPS_ACC_MD%d(d, %s) ob2_chk((d) * ob2_sd%d + %s, ob2_lo%d, ob2_hi%d,"
                      " \"%s\", %d)" % (i, ", ".join(coords), i, expr, i, i, kd.name, i))
                    continue
                w("#define OPS_ACC%d(%s) (%s)" % (i, ", ".join(coords), expr))
                w("#define OPS_ACC_MD%d(d, %s) ((d) * ob2_sd%d + %s)" %
                  (i, ", ".join(coords), i, expr))
            masked = mask_comments_strings(text)
            op = masked.index("(", masked.find(kd.name))
            cl = match_paren(masked, op)
            extra = "".join(", int ob2_sx%d, int ob2_sy%d, int ob2_sz%d, int ob2_sd%d" %
                            (i, i, i, i) for i in idx)
            if self.check:
                extra += "".join(", long long ob2_lo%d, long long ob2_hi%d" % (i, i) for i in idx)
            w("static __device__ __forceinline__ " + text[:cl] + extra + text[cl:])
            for i in idx:
                w("#undef OPS_ACC%d" % i)
                w("#undef OPS_ACC_MD%d" % i)

        if self.check:
            w("static __device__ long long ob2_chk(long long m, long long lo, long long hi,"
              " const char *k, int a) {")
            w("  if (m >= lo && m < hi) return m;")
            w("  printf(\"OPS_B200_CHECK: %s arg %d offset %lld outside [%lld, %lld) at thread"
              " (%d,%d,%d) block (%d,%d,%d)\\n\", k, a, m, lo, hi, (int)threadIdx.x,"
              " (int)threadIdx.y, (int)threadIdx.z, (int)blockIdx.x, (int)blockIdx.y,"
              " (int)blockIdx.z);")
            w("  return lo;")
            w("}")
            w("static __device__ double ob2_dummy[64];")
        emitted = set()
        for h in self.headers:
            if not self.is_kernel_header(h):
                continue
            for kd in top_level_functions(open(h).read(), h):
                if kd.name in emitted:
                    continue
                emitted.add(kd.name)
                emit_fn(kd)
        for loop in self.loops.values():
            if loop.kernel not in self.kernels:
                raise SystemExit("kernel %s not found in the included headers" % loop.kernel)
            if loop.kernel not in emitted:
                emit_fn(self.kernels[loop.kernel])
                emitted.add(loop.kernel)
        for loop in self.loops.values():
            self.emit_loop(loop, w)
        self.emit_fused(w)
        # constant copier
        w("static int ob2_const_copy(const char *name, int dim, int type_size, const char *data,"
          " void *stream) {")
        for c in self.consts.values():
            w('  if (!strcmp(name, "%s")) {' % c.name)
            w("    size_t cap = sizeof(%s);" % c.name)
            w("    size_t n = (size_t)dim * (size_t)type_size;")
            w("    if (n > cap) return -1;")
            w("    return (int)cudaMemcpyToSymbolAsync(%s, data, n, 0, cudaMemcpyHostToDevice,"
              " (cudaStream_t)stream);" % c.name)
            w("  }")
        w("  return 0;")
        w("}")
        w("struct ob2_const_registrar { ob2_const_registrar() {"
          " ob2_register_const_handler(&ob2_const_copy); } };")
        w("static ob2_const_registrar ob2_const_registrar_instance;")
        w("}  // namespace")
        L.insert(1, "/* divisions in user kernels: %d as ob2::div, %d kept as written */" %
                 tuple(self.div_counts) if self.ddiv else
                 "/* divisions in user kernels: all kept as written (OPS_B200_DDIV=0) */")
        with open(os.path.join(self.outdir, self.app + "_kernels.cu"), "w") as f:
            f.write("\n".join(L) + "\n")

    GBL_CAP = 64  # elements kept for a global array whose length is a run-time value

    def gbl_extent(self, dim: str) -> str:
        """The parameter-block extent of an OPS_READ global: its length when
        that is a compile-time expression (literals and macro names), else
        GBL_CAP elements (the stub rejects longer arrays at run time)."""
        d = dim.strip()
        if re.fullmatch(r"[0-9A-Z_\s\*\+\-\(\)]+", d):
            return d
        return str(self.GBL_CAP)

    def emit_fused(self, w) -> None:
        """One kernel that runs several different loops of the application
        in one launch (the runtime passes only loops whose footprints do not
        meet): loop k of the launch takes CTAs [cta0[k], cta0[k+1]) and runs
        the body of loop id[k] on its own parameter block and grid, through
        the body's unrestricted variant."""
        items = self.fuse_items
        w("struct ob2_fuse_params {")
        w("  int n;")
        w("  unsigned cta0[OB2_FUSE_MAX + 1], gx[OB2_FUSE_MAX], gy[OB2_FUSE_MAX];")
        w("  int id[OB2_FUSE_MAX];")
        w("  unsigned off[OB2_FUSE_MAX];")
        w("  alignas(16) char blob[OB2_FUSE_BLOB];")
        w("};")
        lb = "512, %d" % self.minb if self.minb > 0 else "512"
        w("template <bool IDX32>")
        w("__global__ void __launch_bounds__(%s) ob2fk(const __grid_constant__ ob2_fuse_params f) {"
          % lb)
        w("  const unsigned b = blockIdx.x;")
        w("  int i = 0;")
        w("  while (i + 1 < f.n && b >= f.cta0[i + 1]) i++;")
        w("  const unsigned loc = b - f.cta0[i], r = loc / f.gx[i];")
        w("  const unsigned bx = loc - r * f.gx[i], by = r % f.gy[i], bz = r / f.gy[i];")
        w("  const char *prm = f.blob + f.off[i];")
        w("  switch (f.id[i]) {")
        for k, (P, BF) in enumerate(items):
            w("    case %d: %s<false, IDX32>(*(const %s *)prm, bx, by, bz); break;" % (k, BF, P))
        w("    default: break;")
        w("  }")
        w("}")
        w("static int ob2f_launch(int n, const int *ids, const void *const *prm,"
          " const size_t *psz, const unsigned *grids, const unsigned *block, int idx32,"
          " void *st) {")
        w("  if (n < 1 || n > OB2_FUSE_MAX) return (int)cudaErrorInvalidValue;")
        w("  static ob2_fuse_params f;  // host staging (one host thread drives OPS)")
        w("  f.n = n;")
        w("  unsigned long long c = 0;")
        w("  size_t off = 0;")
        w("  for (int k = 0; k < n; k++) {")
        w("    if (ids[k] < 0 || ids[k] >= %d) return (int)cudaErrorInvalidValue;" % len(items))
        w("    off = (off + 15) & ~(size_t)15;")
        w("    if (off + psz[k] > OB2_FUSE_BLOB) return (int)cudaErrorInvalidValue;")
        w("    memcpy(f.blob + off, prm[k], psz[k]);")
        w("    f.off[k] = (unsigned)off;")
        w("    off += psz[k];")
        w("    f.id[k] = ids[k];")
        w("    f.cta0[k] = (unsigned)c;")
        w("    f.gx[k] = grids[3 * k];")
        w("    f.gy[k] = grids[3 * k + 1];")
        w("    c += (unsigned long long)grids[3 * k] * grids[3 * k + 1] * grids[3 * k + 2];")
        w("  }")
        w("  if (c == 0 || c > 0x7fffffffULL) return (int)cudaErrorInvalidValue;")
        w("  f.cta0[n] = (unsigned)c;")
        w("  const dim3 blk(block[0], block[1], block[2]);")
        w("  if (idx32)")
        w("    ob2fk<true><<<(unsigned)c, blk, 0, (cudaStream_t)st>>>(f);")
        w("  else")
        w("    ob2fk<false><<<(unsigned)c, blk, 0, (cudaStream_t)st>>>(f);")
        w("  return (int)cudaGetLastError();")
        w("}")

    ELEM_BYTES = {"double": 8, "long long": 8, "int64_t": 8, "unsigned long long": 8,
                  "float": 4, "int": 4, "unsigned int": 4, "unsigned": 4, "int32_t": 4,
                  "short": 2, "half": 2, "__half": 2, "char": 1, "unsigned char": 1,
                  "bool": 1, "complexd": 16, "complexf": 8}

    def light_y_stencil(self, kd) -> bool:
        """True for a short kernel body (OPS_B200_LIGHT statements at most,
        default 4) that reads a
        neighbour along y, e.g. u(0, 1): consecutive rows handled by one
        thread then share those loads in registers."""
        body = kd.text[kd.text.find("{"):]
        if mask_comments_strings(body).count(";") > self.light_max:
            return False
        return re.search(r"\w\s*\(\s*(?:\d+\s*,\s*)?-?\d+\s*,\s*-?[1-9]\d*\s*[,)]",
                         body) is not None

    def rows_per_thread(self, dats, kd=None) -> int:
        """Points per thread along y.  OPS_B200_PY when set; otherwise 2 for
        a light kernel with a y stencil (register reuse of the shared rows)
        and 1 for the rest.  Loops whose widest dat element is narrower than
        8 bytes take proportionally more rows, so each thread keeps the same
        bytes in flight."""
        base = self.py if self.py_forced else (2 if kd is not None and
                                               self.light_y_stencil(kd) else 1)
        widest = max([self.ELEM_BYTES.get(p.base_type, 8) for i, a, p in dats] or [8])
        return base * max(1, 8 // widest)

    def align_dat(self, loop: Loop, kd, dats, reds, py):
        """3D loops without reductions and with one row per thread: the first
        written one-component dat of 4- or 8-byte elements, on whose rows the
        warps' x ranges are aligned to 128 bytes (rows of dats with halos
        start off that boundary; measured on a write-heavy 3D loop, the ADI
        preproc at 256^3 with 258-element rows: 305 us aligned against
        401-432 us).  None: natural mapping."""
        if reds or loop.ndim != 3 or py != 1 or self.check:
            return None
        for i, a, p in dats:
            if a.acc in ("OPS_WRITE", "OPS_RW", "OPS_INC") and a.dim.strip() == "1" and \
                    not a.prolong and self.ELEM_BYTES.get(p.base_type) in (4, 8):
                return i
        return None

    def tb_candidate(self, loop: Loop, kd):
        """A 2D loop whose only written argument is one dat (OPS_WRITE, one
        component), all other dat arguments read-only, no reductions,
        optional or prolong arguments: its sweeps can be temporally blocked
        (the runtime checks the stencils and the chain).  Returns (index of
        the written argument, indices of the read dats of its element type
        that may be the chain's ping-pong partner) or None."""
        if loop.ndim != 2:
            return None
        ws = []
        for i, (a, p) in enumerate(zip(loop.args, kd.params)):
            if a.kind == "reduce" or (a.kind == "dat" and (a.opt or a.prolong)):
                return None
            if a.kind == "dat" and a.acc != "OPS_READ":
                if a.acc != "OPS_WRITE":
                    return None
                ws.append(i)
        if len(ws) != 1:
            return None
        wi = ws[0]
        wt = kd.params[wi].base_type
        if wt not in ("double", "float") or loop.args[wi].dim.strip() != "1":
            return None
        cand = [i for i, (a, p) in enumerate(zip(loop.args, kd.params))
                if a.kind == "dat" and i != wi and a.acc == "OPS_READ" and p.base_type == wt and
                a.dim.strip() == "1"]
        return (wi, cand) if cand else None

    def emit_tblock(self, loop: Loop, kd, P, K, I, dats, tb, w) -> None:
        """The temporal-blocking kernel of a loop (ob2_tblock in
        ops_b200_loop.h): CTA tile OB2_TB_TX x OB2_TB_TY of the range, region
        widened by `steps` in shared memory, the loop's point function on it
        with the two ping-pong dats' views patched to the shared buffers."""
        wi, cand = tb
        T = kd.params[wi].base_type
        TN = "ob2t_" + loop.stub[len("ops_par_loop_"):]
        w("template <bool IDX32>")
        w("__global__ void __launch_bounds__(256) %sT(const __grid_constant__ %s p,"
          " const __grid_constant__ ob2_tblock t) {" % (K, P))
        w("  extern __shared__ double ob2_tbsm[];")
        w("  __shared__ %s pp;  // the parameters with the two dats' views in shared memory" % P)
        w("  const int S = t.steps, PX = OB2_TB_TX + 2 * S, PY = OB2_TB_TY + 2 * S;")
        w("  %s *buf0 = (%s *)ob2_tbsm, *buf1 = buf0 + PX * PY;" % (T, T))
        w("  const int tid = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;")
        w("  const int tx0 = p.lo0 + (int)blockIdx.x * OB2_TB_TX, ty0 = p.lo1 + (int)blockIdx.y * OB2_TB_TY;")
        w("  const int tx1 = min(tx0 + OB2_TB_TX, p.hi0), ty1 = min(ty0 + OB2_TB_TY, p.hi1);")
        w("  const int X0 = tx0 - S, Y0 = ty0 - S;")
        # the views of X (arg s) and Y (arg wi): element of (x, y) = b + x*wx + y*wy
        w("  const %s *gx = nullptr; int xwx = 0, xwy = 0;" % T)
        for i in cand:
            w("  if (t.s == %d) { gx = p.b%d; xwx = (int)p.wx%d; xwy = (int)p.wy%d; }" % (i, i, i, i))
        w("  %s *gy = p.b%d; const int ywx = (int)p.wx%d, ywy = (int)p.wy%d;" % (T, wi, wi, wi))
        w("  if (tid == 0) {")
        w("    pp = p;")
        for i in cand:
            w("    if (t.s == %d) { pp.wx%d = 1; pp.wy%d = PX; pp.wz%d = 0; pp.ey%d = PX; }" %
              (i, i, i, i, i))
        w("    pp.wx%d = 1; pp.wy%d = PX; pp.wz%d = 0; pp.ey%d = PX;" % (wi, wi, wi, wi))
        w("  }")
        # load: X over the region within the range widened by one, Y outside
        # the range (its values there never change)
        w("  for (int k = tid; k < PX * PY; k += nt) {")
        w("    const int x = X0 + k % PX, y = Y0 + k / PX;")
        w("    if (x < p.lo0 - 1 || x > p.hi0 || y < p.lo1 - 1 || y > p.hi1 || x < t.sx0 ||"
          " x >= t.sx1 || y < t.sy0 || y >= t.sy1) continue;")
        w("    buf0[k] = gx[x * xwx + y * xwy];")
        w("    if (x < p.lo0 || x >= p.hi0 || y < p.lo1 || y >= p.hi1) buf1[k] = gy[x * ywx + y * ywy];")
        w("  }")
        w("  __syncthreads();")
        # the sweeps: sweep st reads buffer (st-1)%2 and writes buffer st%2
        # over the tile widened by S - st, clipped to the range
        w("  for (int st = 1; st <= S; st++) {")
        w("    const int m = S - st;")
        w("    %s *in = (st & 1) ? buf0 : buf1, *out = (st & 1) ? buf1 : buf0;" % T)
        w("    %s *inv = in - (X0 + Y0 * PX), *outv = out - (X0 + Y0 * PX);" % T)
        w("    const int rx0 = max(tx0 - m, p.lo0), rx1 = min(tx1 + m, p.hi0);")
        w("    const int ry0 = max(ty0 - m, p.lo1), ry1 = min(ty1 + m, p.hi1);")
        w("    const int rw = rx1 - rx0, n = rw > 0 && ry1 > ry0 ? rw * (ry1 - ry0) : 0;")
        w("    for (int k = tid; k < n; k += nt) {")
        w("      const int x = rx0 + k % rw, y = ry0 + k / rw;")
        qs = []
        for i, a, pr in dats:
            if i == wi:
                qs.append("outv")
            elif i in cand:
                qs.append("(t.s == %d ? inv : p.b%d)" % (i, i))
            else:
                qs.append("p.b%d" % i)
        w("      %s_A<true>(pp, x, y, 0%s);" % (I, "".join(", " + q for q in qs)))
        w("    }")
        w("    __syncthreads();")
        w("  }")
        # write back: X's values into its spare, Y's in place; the edge
        # CTAs also carry X's points outside the range into the spare
        w("  %s *gs = (%s *)t.spare;" % (T, T))
        w("  const int ex0 = blockIdx.x == 0 ? t.sx0 : tx0, ex1 = tx1 >= p.hi0 ? t.sx1 : tx1;")
        w("  const int ey0 = blockIdx.y == 0 ? t.sy0 : ty0, ey1 = ty1 >= p.hi1 ? t.sy1 : ty1;")
        w("  const int ew = ex1 - ex0, en = ew > 0 && ey1 > ey0 ? ew * (ey1 - ey0) : 0;")
        w("  for (int k = tid; k < en; k += nt) {")
        w("    const int x = ex0 + k % ew, y = ey0 + k / ew;")
        w("    const int gxo = x * xwx + y * xwy;")
        w("    if (x >= p.lo0 && x < p.hi0 && y >= p.lo1 && y < p.hi1) {")
        w("      const int b = (x - X0) + (y - Y0) * PX;")
        w("      gs[gxo] = buf0[b];")
        w("      gy[x * ywx + y * ywy] = buf1[b];")
        w("    } else {")
        w("      gs[gxo] = gx[gxo];")
        w("    }")
        w("  }")
        w("}")
        w("static int %s(const void *prm, const ob2_tblock *t, void *st) {" % TN)
        w("  const %s &p = *(const %s *)prm;" % (P, P))
        w("  if (t->steps < 2 || t->steps > OB2_TB_MAX || !(%s)) return (int)cudaErrorInvalidValue;" %
          " || ".join("t->s == %d" % i for i in cand))
        w("  const size_t sm = (size_t)2 * (OB2_TB_TX + 2 * t->steps) * (OB2_TB_TY + 2 * t->steps) *"
          " sizeof(%s);" % T)
        w("  static bool attr = false;")
        w("  if (!attr) {")
        w("    cudaFuncSetAttribute(%sT<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,"
          " (int)((size_t)2 * (OB2_TB_TX + 2 * OB2_TB_MAX) * (OB2_TB_TY + 2 * OB2_TB_MAX) *"
          " sizeof(%s)));" % (K, T))
        w("    attr = true;")
        w("  }")
        w("  const dim3 g((unsigned)((p.hi0 - p.lo0 + OB2_TB_TX - 1) / OB2_TB_TX),"
          " (unsigned)((p.hi1 - p.lo1 + OB2_TB_TY - 1) / OB2_TB_TY), 1);")
        w("  %sT<true><<<g, dim3(32, 8, 1), sm, (cudaStream_t)st>>>(p, *t);" % K)
        w("  return (int)cudaGetLastError();")
        w("}")

    def emit_loop(self, loop: Loop, w) -> None:
        kd = self.kernels[loop.kernel]
        if len(kd.params) != len(loop.args):
            raise SystemExit("kernel %s takes %d parameters but the loop passes %d arguments" %
                             (loop.kernel, len(kd.params), len(loop.args)))
        nd = loop.ndim
        P = "ob2p_" + loop.stub[len("ops_par_loop_"):]
        K = "ob2k_" + loop.stub[len("ops_par_loop_"):]
        hd = nd >= 4  # 4D / 5D block: the 4th and 5th axes fold into the grid's z
        if hd and not all(p.is_acc for a, p in zip(loop.args, kd.params) if a.kind == "dat"):
            raise SystemExit("%s: %dD loops need ACC<> kernel parameters" % (loop.kernel, nd))
        w("struct %s {" % P)
        w("  int lo0, lo1, lo2, hi0, hi1, hi2;")
        w("  unsigned int *counter;")
        if hd:
            w("  int lo3, hi3, lo4, hi4;")
        reds = []
        for i, (a, p) in enumerate(zip(loop.args, kd.params)):
            if a.kind == "dat":
                w("  %s *b%d; long long wx%d, wy%d, wz%d; int ex%d, ey%d, ez%d, ed%d;" %
                  (p.base_type, i, i, i, i, i, i, i, i))
                if hd:
                    w("  long long wu%d, wv%d; int eu%d, ev%d;" % (i, i, i, i))
                if a.prolong:  # multigrid stride: the loop index is divided by it
                    w("  int mx%d, my%d, mz%d;" % (i, i, i))
                if self.check:
                    w("  long long clo%d, chi%d;" % (i, i))
            elif a.kind == "gbl":
                w("  %s g%d[%s];" % (p.base_type, i, self.gbl_extent(a.dim)))
            elif a.kind == "reduce":
                w("  %s *r%d; %s *part%d; int first%d;" % (p.base_type, i, p.base_type, i, i))
                reds.append((i, a, p))
        w("};")
        # Point function, in two variants: with __restrict__ dat pointers
        # (the common case: no dat is both written and passed twice, so the
        # compiler may batch every load of the point ahead of its stores) and
        # without (aliasing arguments).
        I = "ob2i_" + loop.stub[len("ops_par_loop_"):]
        dats = [(i, a, p) for i, (a, p) in enumerate(zip(loop.args, kd.params)) if a.kind == "dat"]
        for variant, qual in (("R", "__restrict__ "), ("A", "")):
            prm = "".join(", %s *%sq%d" % (p.base_type, qual, i) for i, a, p in dats)
            prm += "".join(", %s *red%d" % (p.base_type, i) for i, a, p in reds)
            # IDX32: element offsets in 32-bit arithmetic (every dat of the
            # launch has fewer than 2^31 elements; decided by the runtime)
            w("template <bool IDX32>")
            w("static __device__ __forceinline__ void %s_%s(const %s &p, int x, int y, int z%s%s) {" %
              (I, variant, P, ", int u, int v" if hd else "", prm))
            call = []
            for i, (a, p) in enumerate(zip(loop.args, kd.params)):
                if a.kind == "dat":
                    ex = "1" if a.dim.strip() == "1" else "p.ex%d" % i
                    if a.prolong:
                        cx, cy, cz = ("(x / p.mx%d)" % i, "(y / p.my%d)" % i, "(z / p.mz%d)" % i)
                    else:
                        cx, cy, cz = "x", "y", "z"
                    if hd:
                        off = ("(IDX32 ? (long long)(x * (int)p.wx%d + y * (int)p.wy%d + z * (int)p.wz%d"
                               " + u * (int)p.wu%d + v * (int)p.wv%d) : x * p.wx%d + y * p.wy%d"
                               " + z * p.wz%d + u * p.wu%d + v * p.wv%d)" %
                               (i, i, i, i, i, i, i, i, i, i))
                    else:
                        off = ("(IDX32 ? (long long)(%s * (int)p.wx%d + %s * (int)p.wy%d + %s * (int)p.wz%d)"
                               " : %s * p.wx%d + %s * p.wy%d + %s * p.wz%d)" %
                               (cx, i, cy, i, cz, i, cx, i, cy, i, cz, i))
                    # only optional arguments can carry a null dat
                    ptr = ("q%d ? q%d + %s : (%s *)0" % (i, i, off, p.base_type)) if a.opt \
                        else "q%d + %s" % (i, off)
                    if p.is_acc and hd:
                        w("  ACC<%s> a%d(%s, %s, p.ey%d, p.ez%d, p.eu%d, p.ev%d, p.ed%d);" %
                          (p.base_type, i, ptr, ex, i, i, i, i, i))
                    elif p.is_acc:
                        w("  ACC<%s> a%d(%s, %s, p.ey%d, p.ez%d, p.ed%d);" %
                          (p.base_type, i, ptr, ex, i, i, i))
                    else:  # OPS_ACCn kernel: the point's pointer (strides below)
                        if self.check and a.opt:  # a disabled argument points at a dummy
                            ptr = "q%d ? q%d + %s : (%s *)ob2_dummy" % (i, i, off, p.base_type)
                        w("  %s *a%d = %s;" % (p.base_type, i, ptr))
                    call.append("a%d" % i)
                elif a.kind == "gbl":
                    call.append("(%s *)p.g%d" % (p.base_type, i))
                elif a.kind == "reduce":
                    call.append("red%d" % i)
                elif a.kind == "idx":
                    call.append("idx")
            if any(a.kind == "idx" for a in loop.args):
                if hd:
                    w("  int idx[%d] = {x, y, z, u%s};" % (nd, ", v" if nd >= 5 else ""))
                else:
                    w("  int idx[3] = {x, y, z};")
            for i, (a, p) in enumerate(zip(loop.args, kd.params)):
                if a.kind == "dat" and not p.is_acc:
                    ex = "1" if a.dim.strip() == "1" else "p.ex%d" % i
                    call.append("%s, p.ey%d, p.ez%d, p.ed%d" % (ex, i, i, i))
            if self.check:
                for i, (a, p) in enumerate(zip(loop.args, kd.params)):
                    if a.kind == "dat" and not p.is_acc:
                        if a.prolong:
                            po = ("((x / p.mx%d) * p.wx%d + (y / p.my%d) * p.wy%d +"
                                  " (z / p.mz%d) * p.wz%d)" % (i, i, i, i, i, i))
                        else:
                            po = "(x * p.wx%d + y * p.wy%d + z * p.wz%d)" % (i, i, i)
                        call.append("p.clo%d - %s, p.chi%d - %s" % (i, po, i, po))
            w("  %s(%s);" % (loop.kernel, ", ".join(call)))
            w("}")
        py = 1 if hd else self.rows_per_thread(dats, kd)
        # a 3D loop whose extra rows per thread come only from its narrow
        # elements (not from stencil reuse along y) takes one row per thread
        # with 128-byte row alignment instead
        if (not hd and loop.ndim == 3 and not reds and py > 1 and not self.py_forced and
                not self.light_y_stencil(kd) and self.align_dat(loop, kd, dats, reds, 1) is not None):
            py = 1
        aw = self.align_dat(loop, kd, dats, reds, py)
        if aw is not None:
            w("template <bool RESTRICT, bool IDX32, bool ALIGN = true>")
        else:
            w("template <bool RESTRICT, bool IDX32>")
        minb = self.minb if not reds else 0
        lb = "512, %d" % minb if minb > 0 else "512"
        BF = "ob2b_" + loop.stub[len("ops_par_loop_"):]
        if reds:
            w("__global__ void __launch_bounds__(%s) %s(const __grid_constant__ %s p) {" %
              (lb, K, P))
            w("  const unsigned bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;")
        else:
            # the body takes its CTA coordinates as arguments, so that one
            # launch can also run several instances of this loop (blocks of a
            # multi-block program) side by side: kernel <K>M below
            w("static __device__ __forceinline__ void %s(const %s &p, unsigned bx, unsigned by,"
              " unsigned bz) {" % (BF, P))
        if aw is None:
            w("  const int x = p.lo0 + (int)(bx * blockDim.x + threadIdx.x);")
        for i, a, p in reds:
            w("  %s red%d[%s];" % (p.base_type, i, a.dim))
            w("  for (int d = 0; d < (%s); d++) red%d[d] = ob2::identity<%s, %s>();" %
              (a.dim, i, p.base_type, a.acc))
        args_call = "".join(", p.b%d" % i for i, a, p in dats) + \
            "".join(", red%d" % i for i, a, p in reds)
        if reds:
            py = max(py, self.rpy)
            # reductions: grid of about one wave of resident CTAs, threads
            # stride over y and z, so that few per-CTA partials are combined;
            # PY strided rows per trip, so that their loads are in flight
            # together
            w("  if (x < p.hi0) {")
            w("    const int ys = (int)(gridDim.y * blockDim.y) * %d;" % py)
            if hd:  # the 3rd to 5th axes as one folded index
                w("    const int nz = p.hi2 - p.lo2, nu = p.hi3 - p.lo3, nzu = nz * (p.hi4 - p.lo4) * nu;")
                w("    for (int zz = (int)(bz * blockDim.z + threadIdx.z); zz < nzu;"
                  " zz += (int)(gridDim.z * blockDim.z)) {")
                w("      const int z = p.lo2 + zz % nz, u = p.lo3 + (zz / nz) % nu,"
                  " v = p.lo4 + zz / (nz * nu);")
            else:
                w("    for (int z = p.lo2 + (int)(bz * blockDim.z + threadIdx.z); z < p.hi2;"
                  " z += (int)(gridDim.z * blockDim.z))")
            w("      for (int yb = p.lo1 + (int)(by * blockDim.y + threadIdx.y) * %d;"
              " yb < p.hi1; yb += ys) {" % py)
            # PY consecutive rows per trip; all in range: no branch between
            # the calls, so the loads of every row can be issued before the
            # stores of the first, and rows shared by the stencils are loaded
            # once
            zc = "z, u, v" if hd else "z"
            w("        if (yb + %d < p.hi1) {" % (py - 1))
            w("#pragma unroll")
            w("          for (int j = 0; j < %d; j++) {" % py)
            w("            if (RESTRICT) %s_R<IDX32>(p, x, yb + j, %s%s);" % (I, zc, args_call))
            w("            else %s_A<IDX32>(p, x, yb + j, %s%s);" % (I, zc, args_call))
            w("          }")
            w("        } else {")
            w("          for (int y = yb; y < p.hi1; y++) {")
            w("            if (RESTRICT) %s_R<IDX32>(p, x, y, %s%s);" % (I, zc, args_call))
            w("            else %s_A<IDX32>(p, x, y, %s%s);" % (I, zc, args_call))
            w("          }")
            w("        }")
            w("      }")
            if hd:
                w("    }")
            w("  }")
        else:
            # PY points per thread along y (consecutive rows), x / z one each
            w("  const int y0 = p.lo1 + (int)(by * blockDim.y + threadIdx.y) * %d;" % py)
            if hd:  # the 3rd to 5th axes as one folded index
                w("  const int nz = p.hi2 - p.lo2, nu = p.hi3 - p.lo3;")
                w("  const int zz = (int)(bz * blockDim.z + threadIdx.z);")
                w("  if (zz >= nz * nu * (p.hi4 - p.lo4)) return;")
                w("  const int z = p.lo2 + zz % nz, u = p.lo3 + (zz / nz) % nu,"
                  " v = p.lo4 + zz / (nz * nu);")
                w("  if (x < p.hi0 && y0 < p.hi1) {")
                w("    if (RESTRICT) %s_R<IDX32>(p, x, y0, z, u, v%s);" % (I, args_call))
                w("    else %s_A<IDX32>(p, x, y0, z, u, v%s);" % (I, args_call))
                w("  }")
            else:
                w("  const int z = p.lo2 + (int)(bz * blockDim.z + threadIdx.z);")
            if hd:
                pass
            elif aw is not None:
                # x starts the row's misalignment (in elements of dat aw)
                # before lo0, so that a warp's accesses to the rows of aw
                # begin on 128-byte boundaries; the grid has that many
                # columns to spare
                i = aw
                es = self.ELEM_BYTES[kd.params[i].base_type]
                w("  const int sh = ALIGN && p.wx%d == 1 ? (int)(((unsigned long long)(p.b%d + "
                  "(long long)p.lo0 + (long long)y0 * p.wy%d + (long long)z * p.wz%d) / %d) & %d)"
                  " : 0;" % (i, i, i, i, es, 128 // es - 1))
                w("  const int x = p.lo0 - sh + (int)(bx * blockDim.x + threadIdx.x);")
                w("  if (x >= p.lo0 && x < p.hi0 && z < p.hi2) {")
            else:
                w("  if (x < p.hi0 && z < p.hi2) {")
            if hd:
                pass
            elif py == 1:
                w("    if (y0 < p.hi1) {")
                w("      if (RESTRICT) %s_R<IDX32>(p, x, y0, z%s);" % (I, args_call))
                w("      else %s_A<IDX32>(p, x, y0, z%s);" % (I, args_call))
                w("    }")
            else:
                # all PY rows in range: no branch between the calls (loads of
                # every row may be issued before the first row's stores)
                w("    if (y0 + %d < p.hi1) {" % (py - 1))
                w("#pragma unroll")
                w("      for (int j = 0; j < %d; j++) {" % py)
                w("        if (RESTRICT) %s_R<IDX32>(p, x, y0 + j, z%s);" % (I, args_call))
                w("        else %s_A<IDX32>(p, x, y0 + j, z%s);" % (I, args_call))
                w("      }")
                w("    } else {")
                w("      for (int y = y0; y < p.hi1; y++) {")
                w("        if (RESTRICT) %s_R<IDX32>(p, x, y, z%s);" % (I, args_call))
                w("        else %s_A<IDX32>(p, x, y, z%s);" % (I, args_call))
                w("      }")
                w("    }")
            if not hd:
                w("  }")
        if reds:
            w("  __shared__ double ob2_sh_raw[32 * 2];")
            w("  __shared__ int ob2_flag;")
            for i, a, p in reds:
                w("  ob2::block_partial<%s, %s>(red%d, %s, p.part%d, (%s *)ob2_sh_raw);" %
                  (p.base_type, a.acc, i, a.dim, i, p.base_type))
            w("  if (ob2::last_block(p.counter, &ob2_flag)) {")
            for i, a, p in reds:
                w("    ob2::final_combine<%s, %s>(%s, p.part%d, p.r%d, p.first%d,"
                  " (%s *)ob2_sh_raw);" % (p.base_type, a.acc, a.dim, i, i, i, p.base_type))
            w("    ob2::reset_counter(p.counter);")
            w("  }")
        w("}")
        if not reds:
            w("template <bool RESTRICT, bool IDX32>")
            w("__global__ void __launch_bounds__(%s) %s(const __grid_constant__ %s p) {" %
              (lb, K, P))
            w("  %s<RESTRICT, IDX32>(p, blockIdx.x, blockIdx.y, blockIdx.z);" % BF)
            w("}")
            # several instances in one launch: instance it takes the grid's z
            # slab [it * gz, (it + 1) * gz); CTAs past an instance's own range
            # find no points
            w("struct %sM { %s p[OB2_MULTI_MAX]; unsigned gz; };" % (P, P))
            w("template <bool RESTRICT, bool IDX32>")
            w("__global__ void __launch_bounds__(%s) %sM(const __grid_constant__ %sM m) {" %
              (lb, K, P))
            w("  const unsigned it = blockIdx.z / m.gz;")
            w("  %s<RESTRICT, IDX32>(m.p[it], blockIdx.x, blockIdx.y, blockIdx.z - it * m.gz);" %
              BF)
            w("}")
            # the same with a halo group folded in: each CTA first copies the
            # group's cells in its footprint (tile widened by the stencil
            # reach), then runs the loop; unrestricted pointers, since the
            # loop reads cells this launch writes
            w("template <bool IDX32>")
            w("__global__ void __launch_bounds__(%s) %sH(const __grid_constant__ %sM m,"
              " const __grid_constant__ ob2_hfuse h) {" % (lb, K, P))
            w("  const unsigned it = blockIdx.z / m.gz, bz = blockIdx.z - it * m.gz;")
            w("  const %s &p = m.p[it];" % P)
            w("  const int x0 = p.lo0 + (int)(blockIdx.x * blockDim.x);")
            w("  const int y0 = p.lo1 + (int)(blockIdx.y * blockDim.y) * %d;" % py)
            w("  const int z0 = p.lo2 + (int)(bz * blockDim.z);")
            w("  ob2::hfuse_prologue(h, (int)it, x0, min(x0 + (int)blockDim.x, p.hi0), y0,"
              " min(y0 + (int)blockDim.y * %d, p.hi1), z0, min(z0 + (int)blockDim.z, p.hi2));" %
              py)
            w("  __syncthreads();")
            w("  %s<false, IDX32%s>(p, blockIdx.x, blockIdx.y, bz);" %
              (BF, ", false" if aw is not None else ""))
            w("}")
        tb = self.tb_candidate(loop, kd)
        if tb:
            self.emit_tblock(loop, kd, P, K, I, dats, tb, w)
        # launchers: the runtime launches a loop now or, in lazy mode, later
        # (possibly once per tile, possibly inside a graph capture)
        LN = "ob2l_" + loop.stub[len("ops_par_loop_"):]
        MN = "ob2m_" + loop.stub[len("ops_par_loop_"):]
        if not reds:
            for rs, ix in (("false", "false"), ("false", "true"), ("true", "false"),
                           ("true", "true")):
                w("static int %s_%s_%s(const void *const *prm, int n, const unsigned *g,"
                  " const unsigned *b, void *st) {" % (MN, rs[0], ix[0]))
                w("  if (n < 1 || n > OB2_MULTI_MAX) return (int)cudaErrorInvalidValue;")
                w("  %sM m;" % P)
                w("  for (int k = 0; k < n; k++) m.p[k] = *(const %s *)prm[k];" % P)
                w("  m.gz = g[2];")
                w("  %sM<%s, %s><<<dim3(g[0], g[1], g[2] * n), dim3(b[0], b[1], b[2]), 0,"
                  " (cudaStream_t)st>>>(m);" % (K, rs, ix))
                w("  return (int)cudaGetLastError();")
                w("}")
        HN = "ob2h_" + loop.stub[len("ops_par_loop_"):]
        if not reds:
            for ix in ("false", "true"):
                w("static int %s_%s(const void *const *prm, int n, const unsigned *g,"
                  " const unsigned *b, const ob2_hfuse *h, void *st) {" % (HN, ix[0]))
                w("  if (n < 1 || n > OB2_MULTI_MAX) return (int)cudaErrorInvalidValue;")
                w("  %sM m;" % P)
                w("  for (int k = 0; k < n; k++) m.p[k] = *(const %s *)prm[k];" % P)
                w("  m.gz = g[2];")
                w("  %sH<%s><<<dim3(g[0], g[1], g[2] * n), dim3(b[0], b[1], b[2]), 0,"
                  " (cudaStream_t)st>>>(m, *h);" % (K, ix))
                w("  return (int)cudaGetLastError();")
                w("}")
        for rs, ix in (("false", "false"), ("false", "true"), ("true", "false"), ("true", "true")):
            w("static int %s_%s_%s(const void *prm, const unsigned *g, const unsigned *b,"
              " void *st) {" % (LN, rs[0], ix[0]))
            w("  %s<%s, %s><<<dim3(g[0], g[1], g[2]), dim3(b[0], b[1], b[2]), 0,"
              " (cudaStream_t)st>>>(*(const %s *)prm);" % (K, rs, ix, P))
            w("  return (int)cudaGetLastError();")
            w("}")
        # host stub
        params = ", ".join("ops_arg arg%d" % i for i in range(len(loop.args)))
        ns = re.sub(r"\W", "_", self.app)
        w("}  // namespace")
        w("void %s(char const *name, ops_block block, int dim, int *range%s) {" %
          (loop.stub, (", " + params) if params else ""))
        w("  using namespace ob2_%s;" % ns)
        na = len(loop.args)
        w("  ops_arg args[%d] = {%s};" % (max(na, 1), ", ".join("arg%d" % i for i in range(na))
                                          or "ops_arg_idx()"))
        w("  ob2_loop L;")
        w("  L.prolong_mask = %du;" % sum(1 << i for i, a in enumerate(loop.args)
                                         if a.kind == "dat" and a.prolong))
        w("  if (!ob2_loop_begin(&L, name, block, dim, range, args, %d)) return;" % na)
        w("  %s p;" % P)
        # zeroed: the block is compared byte for byte (graph replay), so its
        # padding must not carry stack contents
        w("  memset((void *)&p, 0, sizeof(p));")
        w("  p.lo0 = L.lo[0]; p.lo1 = L.lo[1]; p.lo2 = L.lo[2];")
        w("  p.hi0 = L.hi[0]; p.hi1 = L.hi[1]; p.hi2 = L.hi[2];")
        if hd:
            w("  p.lo3 = L.lo4[0]; p.hi3 = L.hi4[0]; p.lo4 = L.lo4[1]; p.hi4 = L.hi4[1];")
        w("  p.counter = L.counter;")
        w("  dim3 blk(L.block[0], L.block[1], L.block[2]);")
        w("  dim3 grd(L.grid[0], L.grid[1], L.grid[2]);")
        if aw is not None:  # the x extent covers a row's misalignment too
            w("  grd.x = (unsigned)((L.n[0] + %d + (int)blk.x - 1) / (int)blk.x);" %
              (128 // self.ELEM_BYTES[kd.params[aw].base_type] - 1))
        if not reds and py > 1:
            w("  grd.y = (L.n[1] + blk.y * %d - 1) / (blk.y * %d);" % (py, py))
        elif reds and py > 1:
            w("  grd.y = std::max(1u, std::min(grd.y, (unsigned)((L.n[1] + blk.y * %d - 1) /"
              " (blk.y * %d))));" % (py, py))
        if reds:
            w("  size_t nblk = (size_t)grd.x * grd.y * grd.z;")
            w("  char *scratch = (char *)L.partials;")
        for i, (a, p) in enumerate(zip(loop.args, kd.params)):
            if a.kind == "dat":
                w("  p.b%d = (%s *)L.view[%d].base; p.wx%d = L.view[%d].wx; p.wy%d = L.view[%d].wy;"
                  " p.wz%d = L.view[%d].wz;" % (i, p.base_type, i, i, i, i, i, i, i))
                w("  p.ex%d = L.view[%d].ex; p.ey%d = L.view[%d].ey; p.ez%d = L.view[%d].ez;"
                  " p.ed%d = L.view[%d].ed;" % (i, i, i, i, i, i, i, i))
                if hd:
                    w("  p.wu%d = L.view[%d].wu; p.wv%d = L.view[%d].wv; p.eu%d = L.view[%d].eu;"
                      " p.ev%d = L.view[%d].ev;" % (i, i, i, i, i, i, i, i))
                if a.prolong:
                    w("  p.mx%d = arg%d.stencil->mgrid_stride[0];" % (i, i))
                    w("  p.my%d = dim > 1 ? arg%d.stencil->mgrid_stride[1] : 1;" % (i, i))
                    w("  p.mz%d = dim > 2 ? arg%d.stencil->mgrid_stride[2] : 1;" % (i, i))
                if self.check:
                    w("  if (arg%d.dat && L.view[%d].base) {" % (i, i))
                    w("    p.clo%d = (long long)((char *)arg%d.dat->data_d - L.view[%d].base) /"
                      " (long long)sizeof(%s);" % (i, i, i, p.base_type))
                    w("    p.chi%d = p.clo%d + (long long)(arg%d.dat->mem / sizeof(%s));" %
                      (i, i, i, p.base_type))
                    w("  } else { p.clo%d = 0; p.chi%d = 0; }" % (i, i))
            elif a.kind == "gbl":
                w("  if ((size_t)arg%d.dim * (size_t)arg%d.elem_size > sizeof(p.g%d))"
                  " throw OPSException(OPS_INVALID_ARGUMENT, \"Error: ops_arg_gbl larger than"
                  " declared in the par_loop\");" % (i, i, i))
                w("  memcpy(p.g%d, arg%d.data, (size_t)arg%d.dim * (size_t)arg%d.elem_size);" %
                  (i, i, i, i))
            elif a.kind == "reduce":
                w("  p.r%d = (%s *)L.red[%d].acc; p.first%d = L.red[%d].first;" %
                  (i, p.base_type, i, i, i))
                w("  p.part%d = (%s *)scratch;"
                  " scratch += ((nblk * (%s) * sizeof(%s) + 255) / 256) * 256;" %
                  (i, p.base_type, a.dim, p.base_type))
        w("  const bool al = ob2_args_alias(args, %d) != 0;" % na)
        w("  const ob2_launcher fn = al ? (L.idx32 ? %s_f_t : %s_f_f)"
          " : (L.idx32 ? %s_t_t : %s_t_f);" % (LN, LN, LN, LN))
        w("  const unsigned g3[3] = {grd.x, grd.y, grd.z}, b3[3] = {blk.x, blk.y, blk.z};")
        if reds:
            w("  const ob2_mlauncher mfn = nullptr;")
        else:
            w("  const ob2_mlauncher mfn = al ? (L.idx32 ? %s_f_t : %s_f_f)"
              " : (L.idx32 ? %s_t_t : %s_t_f);" % (MN, MN, MN, MN))
        if not reds and not hd:
            w("  L.fuse_id = %d;" % len(self.fuse_items))
            w("  L.ffn = ob2f_launch;")
            w("  L.hfn = L.idx32 ? %s_t : %s_f;" % (HN, HN))
            self.fuse_items.append((P, "ob2b_" + loop.stub[len("ops_par_loop_"):]))
        if tb:
            TN = "ob2t_" + loop.stub[len("ops_par_loop_"):]
            offs = ", ".join(("offsetof(%s, b%d)" % (P, i)) if a.kind == "dat" else "0"
                             for i, a in enumerate(loop.args))
            roles = ", ".join("2" if i == tb[0] else ("1" if i in tb[1] else "0")
                              for i in range(len(loop.args)))
            w("  static const size_t tb_off[%d] = {%s};" % (len(loop.args), offs))
            w("  static const int tb_role[%d] = {%s};" % (len(loop.args), roles))
            w("  L.tfn = L.idx32 && !al ? %s : nullptr;" % TN)
            w("  L.tb_off = tb_off;")
            w("  L.tb_role = tb_role;")
        w("  ob2_launch(&L, fn, mfn, &p, sizeof(p), g3, b3, %d);" % (1 if reds else py))
        w("  ob2_loop_end(&L);")
        w("}")
        w("namespace ob2_%s {" % ns)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="OPS -> B200 translator")
    ap.add_argument("sources", nargs="+")
    ap.add_argument("-I", dest="incs", action="append", default=[])
    ap.add_argument("--app", default=None)
    ap.add_argument("--out", default=".")
    a = ap.parse_args(argv)
    app = a.app or os.path.splitext(os.path.basename(a.sources[0]))[0]
    Translator([os.path.abspath(s) for s in a.sources], a.incs, app, a.out).run()
    return 0


if __name__ == "__main__":
    sys.exit(main())
