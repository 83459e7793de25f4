"""Mechanical translation of the reference's compute-shader functions
(a GLSL subset: int/uint scalars and arrays, if/else, for, switch, ternaries)
into Python source, so the shaders' own arithmetic can be run on the CPU to
make golden vectors. Used only by make_golden.py when it generates the
fixtures; the translated code is executed there and never committed.

The translation is statement by statement and deliberately literal: every
statement keeps its operands and order; only syntax changes (braces become
indentation, `/` becomes floor division — every division in the translated
functions has non-negative operands — and casts become calls of the
harness's u32()/i32()/u8()).
"""
import re

_TYPES = r"(?:int|uint|bool|ivec2|uvec2|ivec4|uvec4)"


def extract_function(src, name):
    """(parameter text, body text) of `<type> name(...) { ... }`."""
    m = re.search(r"\b\w+\s+%s\s*\(([^)]*)\)\s*\{" % re.escape(name), src)
    if not m:
        raise ValueError("function %s not found" % name)
    i, depth = m.end(), 1
    while depth:
        depth += (src[i] == "{") - (src[i] == "}")
        i += 1
    return m.group(1), src[m.end():i - 1]


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def _ternary(e):
    """`c ? a : b` at paren depth 0 -> Python conditional expression."""
    depth, q = 0, -1
    for k, ch in enumerate(e):
        depth += (ch == "(") - (ch == ")")
        if ch == "?" and depth == 0:
            q = k
            break
    if q < 0:
        return e
    depth = 0
    for k in range(q + 1, len(e)):
        depth += (e[k] == "(") - (e[k] == ")")
        if e[k] == ":" and depth == 0:
            return "((%s) if (%s) else (%s))" % (_expr(e[q + 1:k]), e[:q].strip(), _expr(e[k + 1:]))
    raise ValueError("unbalanced ternary: %r" % e)


def _expr(e):
    e = e.strip()
    e = re.sub(r"\b(\d+)u\b", r"\1", e)                                  # 128u -> 128
    e = re.sub(r"\.xy\b", "", e)                 # 2-component swizzle: the harness passes 2-tuples
    e = re.sub(r"(\w|\])\.(x|y|z|w)\b", lambda m: "%s[%d]" % (m.group(1), "xyzw".index(m.group(2))), e)
    e = e.replace("&&", " and ").replace("||", " or ")
    e = re.sub(r"!(?!=)", " not ", e)
    e = re.sub(r"\buint8_t\(", "u8(", e)
    e = re.sub(r"\buint\(", "u32(", e)
    e = re.sub(r"\bint\(", "i32(", e)
    e = re.sub(r"\b(?:uvec2|ivec2)\(", "vec2(", e)
    e = re.sub(r"(?<![/])/(?![/=])", "//", e)
    return _ternary(e)


def _tokens(body):
    """Statements (with their `;`) and braces, in order."""
    out, cur, depth = [], "", 0
    for ch in body:
        depth += (ch == "(") - (ch == ")")
        if ch in "{}" and depth == 0:
            if cur.strip():
                out.append(" ".join(cur.split()))
            out.append(ch)
            cur = ""
        elif ch == ";" and depth == 0:
            out.append(" ".join(cur.split()) + ";")
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(" ".join(cur.split()))
    return out


def _head(t, kw):
    """For `kw (...) rest`: (inside of the parentheses, rest), else None."""
    m = re.match(r"^%s\s*\(" % kw, t)
    if not m:
        return None
    depth, k = 1, m.end()
    while depth:
        depth += (t[k] == "(") - (t[k] == ")")
        k += 1
    return t[m.end():k - 1], t[k:].strip()


class _Emitter:
    def __init__(self):
        self.lines = []

    def __call__(self, depth, s):
        self.lines.append("    " * depth + s)


def _block(toks, i, depth, emit, switch=None):
    """Translate statements from toks[i] up to the matching `}` (or one
    statement when the caller has no brace); returns the index after it."""
    while i < len(toks):
        t = toks[i]
        i += 1
        if t == "}":
            return i
        if t == "{":
            i = _block(toks, i, depth, emit, switch)
            continue
        i = _statement(t, toks, i, depth, emit, switch)
    return i


def _body(rest, toks, i, depth, emit, switch):
    """Body of if/for/else: an inline statement, a braced block or the next
    statement."""
    if rest:
        return _statement(rest, toks, i, depth, emit, switch)
    if i < len(toks) and toks[i] == "{":
        return _block(toks, i + 1, depth, emit, switch)
    t = toks[i]
    return _statement(t, toks, i + 1, depth, emit, switch)


def _statement(t, toks, i, depth, emit, switch):
    h = _head(t, "if")
    if h:
        emit(depth, "if %s:" % _expr(h[0]))
        i = _body(h[1], toks, i, depth + 1, emit, switch)
        while i < len(toks) and toks[i].startswith("else"):
            t2 = toks[i]
            i += 1
            h2 = _head(t2[4:].strip(), "if")
            if h2:
                emit(depth, "elif %s:" % _expr(h2[0]))
                i = _body(h2[1], toks, i, depth + 1, emit, switch)
            else:
                emit(depth, "else:")
                i = _body(t2[4:].strip(), toks, i, depth + 1, emit, switch)
        return i
    h = _head(t, "for")
    if h:
        m = re.match(r"^\s*(?:%s\s+)?(\w+)\s*=\s*([^;]+);\s*\1\s*<\s*([^;]+);\s*\1\+\+\s*$" % _TYPES, h[0])
        if not m:
            raise ValueError("unsupported for: %r" % t)
        emit(depth, "for %s in range(%s, %s):" % (m.group(1), _expr(m.group(2)), _expr(m.group(3))))
        return _body(h[1], toks, i, depth + 1, emit, switch)
    h = _head(t, "switch")
    if h:
        assert toks[i] == "{"
        i += 1
        var = _expr(h[0])
        first = True
        # cases: label, then statements until the next label or the closing brace
        while toks[i] != "}":
            t2 = toks[i]
            m = re.match(r"^(?:case\s+(\d+)|default)\s*:\s*(.*)$", t2)
            if not m:
                raise ValueError("statement outside a case: %r" % t2)
            i += 1
            if m.group(1) is None:
                emit(depth, "else:")
            else:
                emit(depth, "%s %s == %s:" % ("if" if first else "elif", var, m.group(1)))
            first = False
            emit(depth + 1, "pass")
            if m.group(2):
                i = _statement(m.group(2), toks, i, depth + 1, emit, var)
            while toks[i] != "}" and not re.match(r"^(?:case\s+\d+|default)\s*:", toks[i]):
                if toks[i] == "{":
                    i = _block(toks, i + 1, depth + 1, emit, var)
                else:
                    i = _statement(toks[i], toks, i + 1, depth + 1, emit, var)
        return i + 1
    if t == "break;":
        emit(depth, "pass")
        return i
    if t == "return;":
        emit(depth, "return")
        return i
    if t.startswith("return "):
        emit(depth, "return " + _expr(t[len("return "):-1]))
        return i
    m = re.match(r"^(?:%s)\s+(\w+)\[(\d+)\]\s*;$" % _TYPES, t)
    if m:
        emit(depth, "%s = [0] * %s" % (m.group(1), m.group(2)))
        return i
    m = re.match(r"^(?:%s)\s+(\w+)\s*;$" % _TYPES, t)
    if m:
        emit(depth, "%s = 0" % m.group(1))
        return i
    m = re.match(r"^(?:const\s+)?(?:%s|[A-Z]\w*)\s+(\w+)\s*=\s*(.*);$" % _TYPES, t)
    if m:
        emit(depth, "%s = %s" % (m.group(1), _expr(m.group(2))))
        return i
    m = re.match(r"^(.+?)\s*(\+=|-=|=)\s*(.*);$", t)
    if m:
        emit(depth, "%s %s %s" % (_expr(m.group(1)), m.group(2), _expr(m.group(3))))
        return i
    raise ValueError("untranslated statement: %r" % t)


def translate(src, name, pyname=None):
    """Python source of the GLSL function `name` from shader source `src`."""
    params, body = extract_function(strip_comments(src), name)
    args = [re.sub(r"\[.*\]", "", p.split()[-1]) for p in params.split(",") if p.strip()]
    emit = _Emitter()
    emit(0, "def %s(%s):" % (pyname or name, ", ".join(args)))
    emit(1, "pass")
    _block(_tokens(body) + ["}"], 0, 1, emit)
    return "\n".join(emit.lines) + "\n"
