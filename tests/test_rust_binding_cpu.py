"""The Rust binding (sentinel-x_b200/rust/sxhmm-sys) against the C header:
every function include/sxhmm.h declares is bound with the same parameter
and return types, every struct has the header's fields in the header's
order with the same types, and the constants agree.  No Rust toolchain
exists in this image, so the crate is checked by reading both sources."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sxhmm.h")
CRATE = os.path.join(ROOT, "sentinel-x_b200", "rust", "sxhmm-sys", "src", "lib.rs")

SCALAR = {"int32_t": "i32", "uint32_t": "u32", "int64_t": "i64", "size_t": "usize", "float": "f32",
          "double": "f64", "int": "c_int", "char": "c_char", "uint8_t": "u8", "void": "()"}


def _strip_comments(s):
    return re.sub(r"/\*.*?\*/", "", s, flags=re.S)


def c_to_rust(ctype):
    """A C parameter / field type of the header in Rust spelling."""
    t = " ".join(ctype.replace("*", " * ").split())
    # pointer levels from the right: "const X * const *" -> *const *const X
    parts = t.split("*")
    base = parts[0].strip()
    quals = [q.strip() for q in parts[1:]]
    const_base = base.startswith("const ")
    base = base.replace("const ", "").strip()
    rust = SCALAR.get(base, base)
    if not quals:
        return rust
    # the pointee of the innermost pointer is const if the base is const
    levels = []
    for i, q in enumerate(quals):
        pointee_const = const_base if i == 0 else (quals[i - 1] == "const")
        levels.append("*const " if pointee_const else "*mut ")
    return "".join(reversed(levels)) + rust


def header_functions():
    s = _strip_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"^([A-Za-z_][\w\s\*]*?)\b(sx_\w+)\s*\(([^;]*?)\)\s*;", s, flags=re.M):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3).strip()
        params = []
        if args and args != "void":
            for a in args.split(","):
                a = " ".join(a.split())
                mm = re.match(r"(.*?)(\w+)$", a)
                params.append(c_to_rust(mm.group(1).strip()))
        out[name] = (c_to_rust(ret), params)
    return out


def header_structs():
    s = _strip_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", s, flags=re.S):
        fields = []
        for decl in m.group(1).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            mm = re.match(r"(.*?)\s*((?:\*?\s*\w+(?:\[\d+\])?\s*,\s*)*\*?\s*\w+(?:\[\d+\])?)$", decl)
            base = mm.group(1)
            for nm in mm.group(2).split(","):
                nm = nm.strip()
                stars = nm.count("*")
                nm = nm.replace("*", "").strip()
                arr = re.match(r"(\w+)\[(\d+)\]", nm)
                ty = c_to_rust(base + " *" * stars)
                if arr:
                    fields.append((arr.group(1), f"[{ty}; {arr.group(2)}]"))
                else:
                    fields.append((nm, ty))
        out[m.group(2)] = fields
    return out


def crate_functions():
    s = open(CRATE).read()
    block = s[s.index('extern "C" {'):]
    block = block[:block.index("\n    }\n")]
    out = {}
    for m in re.finditer(r"pub fn (sx_\w+)\((.*?)\)\s*(?:->\s*([^;]+))?;", block, flags=re.S):
        name, args, ret = m.group(1), m.group(2), (m.group(3) or "()").strip()
        params = []
        for a in re.split(r",(?![^\[]*\])", args):
            a = " ".join(a.split())
            if a:
                params.append(a.split(":", 1)[1].strip())
        out[name] = (ret, params)
    return out


def crate_structs():
    s = open(CRATE).read()
    out = {}
    for m in re.finditer(r"pub struct (sx_\w+) \{(.*?)\n    \}", s, flags=re.S):
        fields = []
        for line in m.group(2).split("\n"):
            line = line.strip().rstrip(",")
            mm = re.match(r"pub (\w+): (.+)$", line)
            if mm:
                fields.append((mm.group(1), mm.group(2).strip()))
        if fields:
            out[m.group(1)] = fields
    return out


def test_every_header_function_is_bound_with_its_types():
    h = header_functions()
    r = crate_functions()
    assert len(h) >= 30
    assert set(h) == set(r), (sorted(set(h) - set(r)), sorted(set(r) - set(h)))
    for name, (ret, params) in h.items():
        rret, rparams = r[name]
        assert rret == ret, (name, rret, ret)
        assert rparams == params, (name, rparams, params)


def test_every_header_struct_has_the_same_fields():
    h = header_structs()
    r = crate_structs()
    assert set(h) == set(r), (sorted(set(h) ^ set(r)))
    for name, fields in h.items():
        assert r[name] == fields, (name, r[name], fields)


def test_constants_agree():
    s = open(HEADER).read()
    c = open(CRATE).read()
    consts = re.findall(r"#define (SX_\w+) (\d+)u?", s)
    assert len(consts) >= 15
    for name, val in consts:
        m = re.search(rf"pub const {name}: \w+ = (\d+);", c)
        assert m and int(m.group(1)) == int(val), name
