"""The openmvg-ba-cuda Rust shim (openmvg-rs_b200/rust/openmvg-ba-cuda) cannot be compiled here (no
Rust toolchain), so its raw bindings are checked as text against include/ba_cuda.h: every struct the
shim mirrors has the header's fields in the header's order with matching scalar types, and every
function the shim declares is declared by the header."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ba_cuda.h")
FFI = os.path.join(ROOT, "openmvg-rs_b200", "rust", "openmvg-ba-cuda", "src", "ffi.rs")

C_TO_RUST = {"int32_t": "i32", "uint32_t": "u32", "uint64_t": "u64", "double": "f64", "char": "c_char",
             "void*": "*mut c_void"}


def c_structs(text):
    out = {}
    for name, body in re.findall(r"typedef struct (\w+) \{(.*?)\} \1;", text, re.S):
        fields = []
        for line in body.splitlines():
            line = re.sub(r"/\*.*?\*/", "", line).strip()
            if not line or line.startswith("/*") or line.startswith("*"):
                continue
            m = re.match(r"(const\s+)?([\w]+)\s*(\*?)\s*(.+);", line)
            if not m:
                continue
            const, ctype, star, names = m.groups()
            for nm in names.split(","):
                nm = nm.strip()
                arr = re.match(r"(\w+)\[(\d+)\]", nm)
                if arr:
                    fields.append((arr.group(1), ctype, star, int(arr.group(2)), bool(const)))
                else:
                    fields.append((nm.lstrip("*"), ctype, star or ("*" if nm.startswith("*") else ""), 0,
                                   bool(const)))
        out[name] = fields
    return out


def rust_structs(text):
    out = {}
    for name, body in re.findall(r"pub struct (\w+) \{(.*?)\n\}", text, re.S):
        out[name] = re.findall(r"pub (\w+): ([^,]+),", body)
    return out


def test_shim_structs_mirror_the_header():
    c = c_structs(open(HEADER).read())
    rust = rust_structs(open(FFI).read())
    mirrored = ["omvgba_error", "omvgba_pose", "omvgba_intrinsic", "omvgba_problem", "omvgba_config",
                "omvgba_report", "omvgba_solution", "omvgba_preflight", "omvgba_landmark_tracks",
                "omvgba_refresh_result", "omvgba_sfm_workspace", "omvgba_sfm_prepare_config", "omvgba_sfm_prepared"]
    for name in mirrored:
        assert name in c and name in rust, name
        cf, rf = c[name], rust[name]
        assert [f[0] for f in cf] == [f[0] for f in rf], name
        for (fname, ctype, star, count, const), (_, rtype) in zip(cf, rf):
            rtype = rtype.strip()
            if count:
                assert rtype == f"[{C_TO_RUST[ctype]}; {count}]", (name, fname, rtype)
            elif star:
                ptr = "*const" if const else "*mut"
                target = C_TO_RUST.get(ctype, ctype)
                if ctype == "void":
                    target = "c_void"
                if ctype == "uint8_t":
                    target = "u8"
                assert rtype == f"{ptr} {target}", (name, fname, rtype)
            else:
                assert rtype == C_TO_RUST.get(ctype, ctype), (name, fname, rtype)


def test_shim_functions_are_declared_by_the_library():
    header = open(HEADER).read()
    ffi = open(FFI).read()
    block = ffi[ffi.index('unsafe extern "C" {'):]
    for fn in re.findall(r"pub fn (omvgba_\w+)\(", block):
        if fn == "omvgba_struct_sizes":  # exported for bindings, checked by test_abi
            continue
        assert re.search(rf"\b{fn}\(", header), fn
