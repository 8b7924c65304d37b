#!/usr/bin/env python3
"""OKL -> C++ translator for the oracle build (test infrastructure, not product code).

The reference's device code is written in OCCA's OKL kernel language
(cpp/okl/WaveKernels.okl, cpp/okl/WaveKernelsWADG.okl).  OCCA itself is not
available here, so this script performs the same source-to-source rewrite
that OCCA's Serial/OpenMP backend performs, producing plain C++ that the
``occa.hpp`` shim in ``oracle/shim`` JIT-compiles with the host compiler:

* ``for(init; cond; inc; outer0)``  -> an OpenMP ``parallel for`` loop,
* ``for(init; cond; inc; innerN)``  -> a plain serial loop; every
  barrier-delimited inner-loop nest therefore runs to completion before the
  next one starts, which is exactly the semantics the barriers encode,
* ``shared`` arrays                 -> locals of the outer-loop body,
* ``exclusive`` variables           -> arrays indexed by the linear id of the
  (inner1, inner0) iteration, so a value written in one nest is read back by
  the same logical thread in a later nest,
* ``barrier(localMemFence)``        -> removed (the nest split is the barrier),
* ``occaUnroll(n)``                 -> removed.

The translated kernels keep the reference's loop and summation order; only
the control structure is rewritten.  The source files are read from the
reference checkout at build time and the output goes to ``oracle/_ref``;
no reference source is stored in this repository.

Two defects of the shipped sources are handled by extracting kernels one by
one instead of compiling whole files: ``matvec_example``
(cpp/okl/WaveKernels.okl:15-41) is never closed, and a stray ``#endif``
(cpp/okl/WaveKernelsWADG.okl:2439) closes nothing at the end of
rk_surface_planar.  OCCA's own preprocessor accepted that kernel (the
reference launches it every curvilinear stage); an unmatched ``#endif`` in
an extracted kernel body is dropped here.

Usage: okl2c.py SRC.okl OUT.cpp kernel_name [kernel_name ...]
"""
import re
import sys

TOKEN_RE = re.compile(
    r"(?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?[fFuUlL]*)"
    r"|(?P<id>[A-Za-z_]\w*)"
    r"|(?P<other>.)",
    re.S,
)

EXCL_STRIDE = 1024   # max inner0 extent per inner1 index
EXCL_SLOTS = 8 * EXCL_STRIDE  # supports Kblk <= 8


def strip_comments(src):
    out, i, n = [], 0, len(src)
    while i < n:
        if src.startswith("//", i):
            j = src.find("\n", i)
            i = n if j < 0 else j
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(src[i])
            i += 1
    return "".join(out)


def match_close(s, i, open_ch, close_ch):
    """Index of the bracket closing the one at s[i]."""
    depth = 0
    for j in range(i, len(s)):
        if s[j] == open_ch:
            depth += 1
        elif s[j] == close_ch:
            depth -= 1
            if depth == 0:
                return j
    raise ValueError("unbalanced %s%s" % (open_ch, close_ch))


def split_top(s, sep):
    parts, depth, cur = [], 0, []
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur))
    return parts


def extract_kernel(src, name):
    m = re.search(r"\bkernel\s+void\s+%s\s*\(" % re.escape(name), src)
    if not m:
        raise KeyError(name)
    p0 = m.end() - 1
    p1 = match_close(src, p0, "(", ")")
    params = src[p0 + 1:p1]
    b0 = src.index("{", p1)
    b1 = match_close(src, b0, "{", "}")
    return params, src[b0 + 1:b1]


def parse_params(params):
    out = []
    for p in split_top(params, ","):
        p = " ".join(p.split())
        if not p:
            continue
        toks = re.findall(r"[A-Za-z_]\w*|\*", p)
        pname = toks[-1]
        if "*" in toks:
            kind = "ptr"
        elif "int" in toks:
            kind = "int"
        else:
            kind = "real"
        out.append((p, pname, kind))
    return out


def loop_var(init):
    m = re.search(r"([A-Za-z_]\w*)\s*=", init)
    return m.group(1) if m else "0"


def rewrite_loops(body):
    """Rewrite OKL 4-clause for loops; insert the exclusive-slot id at the
    top of every inner0 body."""
    out, i, inner1 = [], 0, []
    # stack of (close_brace_index_in_source, var) for inner1 scopes
    n = len(body)
    while i < n:
        m = re.compile(r"\bfor\s*\(").search(body, i)
        if not m:
            out.append(body[i:])
            break
        out.append(body[i:m.start()])
        # pop inner1 scopes that ended before this loop
        inner1 = [(end, v) for (end, v) in inner1 if end > m.start()]
        p0 = m.end() - 1
        p1 = match_close(body, p0, "(", ")")
        parts = split_top(body[p0 + 1:p1], ";")
        if len(parts) == 4:
            tag = parts[3].strip()
            header = "for(%s;%s;%s)" % (parts[0], parts[1], parts[2])
            b0 = body.index("{", p1)
            b1 = match_close(body, b0, "{", "}")
            if tag.startswith("outer"):
                out.append("OKL_OMP_FOR\n    " + header + body[p1 + 1:b0 + 1])
            elif tag == "inner1":
                inner1.append((b1, loop_var(parts[0])))
                out.append(header + body[p1 + 1:b0 + 1])
            elif tag == "inner0":
                v1 = inner1[-1][1] if inner1 else "0"
                out.append(header + body[p1 + 1:b0 + 1])
                out.append(" const int __eid = (%s)*%d + (%s);"
                           % (v1, EXCL_STRIDE, loop_var(parts[0])))
            else:
                raise ValueError("unknown loop tag " + tag)
            i = b0 + 1
        else:
            out.append(body[m.start():p1 + 1])
            i = p1 + 1
    return "".join(out)


def rewrite_exclusive(body):
    names = []

    def decl(m):
        typ_and_names = " ".join(m.group(1).split())
        toks = split_top(typ_and_names, ",")
        first = toks[0].split()
        typ, rest = " ".join(first[:-1]), [first[-1]] + [t.strip() for t in toks[1:]]
        out = []
        for nm in rest:  # a name may carry array dimensions: one copy per slot
            base, dims = (nm[:nm.index("[")], nm[nm.index("["):]) if "[" in nm else (nm, "")
            names.append(base.strip())
            out.append("%s %s[%d]%s;" % (typ, base.strip(), EXCL_SLOTS, dims))
        return " ".join(out)

    body = re.sub(r"\bexclusive\s+([^;]+);", decl, body)
    if not names:
        return body
    keep = set(names)
    out = []
    decl_re = re.compile(r"\[%d\]" % EXCL_SLOTS)
    for line in body.split("\n"):
        if decl_re.search(line):
            out.append(line)
            continue
        pieces = []
        for t in TOKEN_RE.finditer(line):
            if t.group("id") and t.group("id") in keep:
                pieces.append("%s[__eid]" % t.group("id"))
            else:
                pieces.append(t.group(0))
        out.append("".join(pieces))
    return "\n".join(out)


def drop_unmatched_endif(body):
    """Remove #endif lines that close no #if inside the kernel body."""
    out, depth = [], 0
    for ln in body.split("\n"):
        d = ln.strip()
        if re.match(r"#\s*if", d):
            depth += 1
        elif re.match(r"#\s*endif", d):
            if depth == 0:
                continue
            depth -= 1
        out.append(ln)
    return "\n".join(out)


def translate(src_path, out_path, names):
    src = strip_comments(open(src_path).read())
    chunks = [
        "// Generated by oracle/okl2c.py from %s; do not edit.\n" % src_path.split("/cpp/")[-1],
        "#include \"okl_prelude.h\"\n",
    ]
    for name in names:
        params, body = extract_kernel(src, name)
        plist = parse_params(params)
        body = drop_unmatched_endif(body)
        body = rewrite_exclusive(body)
        body = rewrite_loops(body)
        body = re.sub(r"\bshared\s+", "", body)
        body = re.sub(r"\bbarrier\s*\(\s*localMemFence\s*\)\s*;", ";", body)
        body = re.sub(r"\boccaUnroll\s*\([^)]*\)", "", body)
        body = re.sub(r"\brestrict\b", "__restrict__", body)
        sig = ", ".join(re.sub(r"\brestrict\b", "__restrict__", p) for p, _, _ in plist)
        call = []
        for idx, (p, pname, kind) in enumerate(plist):
            if kind == "ptr":
                ctype = p[: p.rfind(pname)].replace("restrict", "").strip()
                call.append("(%s)a[%d].p" % (ctype, idx))
            elif kind == "int":
                call.append("a[%d].i" % idx)
            else:
                call.append("(dfloat)a[%d].f" % idx)
        chunks.append(
            "#ifdef OKL_WANT_%s\n"
            "static void okl_kernel_%s(%s){%s}\n"
            "extern \"C\" void okl_call_%s(const okl_arg *a){ okl_kernel_%s(%s); }\n"
            "extern \"C\" int okl_nargs_%s(void){ return %d; }\n"
            "#endif\n" % (name, name, sig, body, name, name, ", ".join(call), name, len(plist))
        )
    with open(out_path, "w") as f:
        f.write("\n".join(chunks))


if __name__ == "__main__":
    if len(sys.argv) < 4:
        sys.exit(__doc__)
    translate(sys.argv[1], sys.argv[2], sys.argv[3:])
