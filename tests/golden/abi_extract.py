"""ABI facts of a C header set, as the C compiler sees them: the prototype of
every function it declares (gcc -aux-info, parameter names dropped, typedef
names kept) and the value of every TAPP_* / TPRIMS_* / kDL* constant (enum
members and integer #defines, printed by a small program compiled against the
headers), plus the sizes of the DLPack structs.

make_abi_golden.py runs this on the reference's pinned headers
(crates/tprims-capi/include/tapp.h and tprims/tprims.h) and writes
tests/golden/tapp_abi.json; tests/test_abi_cpu.py runs it on
include/tprims_b200.h and compares, so that a drift of any prototype, enum
value or status code from the reference's headers fails on the CPU."""
import os
import re
import subprocess
import tempfile

NAME = re.compile(r"\b((?:TAPP|TPRIMS|kDL)[A-Za-z0-9_]*)\b")


def _constants(text):
    """Names of enum members and integer #defines in a header's text."""
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    names = set()
    for body in re.findall(r"enum\s*[A-Za-z_0-9]*\s*\{([^}]*)\}", text):
        for item in body.split(","):
            m = re.match(r"\s*([A-Za-z_][A-Za-z0-9_]*)", item)
            if m:
                names.add(m.group(1))
    for m in re.finditer(r"^\s*#\s*define\s+([A-Za-z_][A-Za-z0-9_]*)\s+\(?-?\d+[uUlL]*\)?\s*$", text, re.M):
        names.add(m.group(1))
    return sorted(n for n in names if NAME.fullmatch(n))


def extract(include_dirs, headers, header_files):
    """include_dirs: -I directories; headers: the #include lines' names;
    header_files: the paths whose text is scanned for constant names."""
    text = ""
    for p in header_files:
        with open(p) as f:
            text += f.read() + "\n"
    consts = _constants(text)
    inc = "".join(f"#include <{h}>\n" for h in headers)
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "abi.c")
        with open(src, "w") as f:
            f.write(inc + "#include <stdio.h>\n#include <stddef.h>\nint main(void) {\n")
            for c in consts:
                f.write(f'  printf("%s %lld\\n", "{c}", (long long)({c}));\n')
            for s in ("DLTensor", "DLDevice", "DLDataType"):
                f.write(f'  printf("sizeof({s}) %zu\\n", sizeof({s}));\n')
            f.write("  return 0;\n}\n")
        flags = ["-std=c11"] + [f"-I{d}" for d in include_dirs]
        aux = os.path.join(td, "aux.txt")
        subprocess.run(["gcc", *flags, "-fsyntax-only", "-aux-info", aux, src], check=True, capture_output=True)
        exe = os.path.join(td, "abi")
        subprocess.run(["gcc", *flags, src, "-o", exe], check=True, capture_output=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
        with open(aux) as f:
            aux_lines = f.read().splitlines()
    values = {}
    for line in out.splitlines():
        k, v = line.rsplit(" ", 1)
        values[k] = int(v)
    protos = {}
    for line in aux_lines:
        m = re.match(r"/\*.*?\*/\s*extern\s+(.*?)\s*\b((?:TAPP|tprims)_[A-Za-z0-9_]*)\s*\((.*)\);\s*$", line)
        if m:
            ret = re.sub(r"\s+", " ", m.group(1)).strip()
            args = [re.sub(r"\s+", " ", a).strip() for a in m.group(3).split(",")]
            protos[m.group(2)] = {"ret": ret, "args": args}
    return {"prototypes": protos, "values": values}
