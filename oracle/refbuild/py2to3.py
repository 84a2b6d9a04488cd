"""Mechanical Python-2 -> Python-3 conversion of the reference's kernel
generator (genDT.py, genAlg.py), written for building oracle/_ref.

Test infrastructure only: it rewrites a copy of the generator so that the
reference's own kernels can be generated and compiled here; nothing in the
product imports it.  The rewrite is token-based (the standard tokenize module
reads Python-2 source), so string contents are never touched:

  * print statements -> print() calls (">>f," -> file=f, a trailing comma ->
    end=" ", the soft-space of Python 2);
  * the binary operator "/" -> "//" (every division in the generator is an
    integer index or a %d argument, whose Python-2 result is the floor);
  * the lambdas with a tuple parameter (genAlg.py:257,269) take two
    parameters and map() gets the two sequences instead of their zip();
  * map() returns a list and reduce() comes from functools (a prelude);
  * the two loops that pop and insert keys of data.Registers while iterating
    it (genAlg.py:462-468, 490-496) iterate a snapshot of the keys.  Python 3
    refuses the mutation; Python 2 iterated its hash-slot order, so the order
    in which matching keys were visited is not reproducible.  The recipe
    therefore also generates with the snapshot reversed and checks that both
    orders give the same kernels (refgen_check in the Makefile).

Usage: python py2to3.py <in.py> <out.py>
"""
import io
import sys
import tokenize

PRELUDE = (
    "import builtins as _bi\n"
    "from functools import reduce\n"
    "def map(*a):\n"
    "    return list(_bi.map(*a))\n"
    "import os as _os\n"
    "_SNAPSHOT_ORDER = _os.environ.get('REFGEN_ORDER', 'forward')\n"
    "def _snapshot(d):\n"
    "    k = list(d)\n"
    "    return k[::-1] if _SNAPSHOT_ORDER == 'reversed' else k\n"
)

TUPLE_LAMBDA = ('map( lambda (sign,xyz): " %s %s"%(sign, "dif%s[%d]"%(xyz,uniqdifN)), zip((signx,signy,signz),\'xyz\') )',
                'map( lambda sign,xyz: " %s %s"%(sign, "dif%s[%d]"%(xyz,uniqdifN)), (signx,signy,signz),\'xyz\' )')
MUTATING_LOOP = ("for Sother in data.Registers:", "for Sother in _snapshot(data.Registers):")


def _offsets(src):
    starts, pos = [0], 0
    for line in src.splitlines(keepends=True):
        pos += len(line)
        starts.append(pos)
    return lambda rc: starts[rc[0] - 1] + rc[1]


def convert(src):
    toks = list(tokenize.generate_tokens(io.StringIO(src).readline))
    off = _offsets(src)
    edits = []
    sig = [t for t in toks if t.type not in (tokenize.NL, tokenize.COMMENT)]
    for n, t in enumerate(sig):
        if t.type == tokenize.OP and t.string == "/":
            edits.append((off(t.start), off(t.end), "//"))
            continue
        if not (t.type == tokenize.NAME and t.string == "print"):
            continue
        prev = sig[n - 1] if n > 0 else None
        if prev is not None and not (prev.type in (tokenize.NEWLINE, tokenize.INDENT, tokenize.DEDENT) or
                                     (prev.type == tokenize.OP and prev.string in (":", ";"))):
            continue
        depth, m = 0, n + 1
        while m < len(sig):
            u = sig[m]
            if u.type == tokenize.OP and u.string in "([{":
                depth += 1
            elif u.type == tokenize.OP and u.string in ")]}":
                depth -= 1
            elif depth == 0 and (u.type in (tokenize.NEWLINE, tokenize.ENDMARKER) or
                                 (u.type == tokenize.OP and u.string == ";")):
                break
            m += 1
        args = sig[n + 1:m]
        dest = None
        if args and args[0].type == tokenize.OP and args[0].string == ">>":
            depth, q = 0, 1
            while q < len(args):
                u = args[q]
                if u.type == tokenize.OP and u.string in "([{":
                    depth += 1
                elif u.type == tokenize.OP and u.string in ")]}":
                    depth -= 1
                elif depth == 0 and u.type == tokenize.OP and u.string == ",":
                    break
                q += 1
            dest = src[off(args[1].start):off(args[q - 1].end)]
            args = args[q + 1:]
        soft = bool(args) and args[-1].type == tokenize.OP and args[-1].string == ","
        if soft:
            args = args[:-1]
        body = src[off(args[0].start):off(args[-1].end)] if args else ""
        # divisions inside the arguments are rewritten here, the outer edit replaces them
        inner = [(off(u.start), off(u.end)) for u in args if u.type == tokenize.OP and u.string == "/"]
        if args:
            base = off(args[0].start)
            for a, b in sorted(inner, reverse=True):
                body = body[:a - base] + "//" + body[b - base:]
        parts = [body] if body else []
        if soft:
            parts.append('end=" "')
        if dest is not None:
            parts.append("file=" + dest)
        end = off(sig[m - 1].end) if m - 1 > n else off(t.end)
        edits.append((off(t.start), end, "print(" + ", ".join(parts) + ")"))
    # drop the division edits that lie inside a rewritten print statement
    spans = [(a, b) for a, b, r in edits if r.startswith("print(")]
    edits = [e for e in edits if e[2].startswith("print(") or not any(a <= e[0] < b for a, b in spans)]
    out = src
    for a, b, r in sorted(edits, reverse=True):
        out = out[:a] + r + out[b:]
    return out


def main(inp, outp):
    src = open(inp).read()
    n_lambda = src.count(TUPLE_LAMBDA[0])
    n_loop = src.count(MUTATING_LOOP[0])
    out = convert(src)
    # the exact-text fixes are applied after the token rewrite, which leaves
    # these strings alone (no print, no division inside them)
    out = out.replace(TUPLE_LAMBDA[0], TUPLE_LAMBDA[1]).replace(MUTATING_LOOP[0], MUTATING_LOOP[1])
    if "genAlg" in inp and (n_lambda < 2 or n_loop != 2):
        sys.exit("py2to3: unexpected generator source (%d tuple lambdas, %d mutating loops)" % (n_lambda, n_loop))
    lines = out.splitlines(keepends=True)
    head = 0
    while head < len(lines) and (lines[head].startswith("#!") or "coding" in lines[head]):
        head += 1
    out = "".join(lines[:head]) + PRELUDE + "".join(lines[head:])
    compile(out, outp, "exec")
    open(outp, "w").write(out)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
