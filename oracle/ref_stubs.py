"""oracle/ref_stubs.py -- TEST INFRASTRUCTURE ONLY.

Builds oracle/_ref/libgalpy_ref.so from the reference's own C sources (never
copied into this repository; read where they lie).  The reference's orbit
drivers name ~45 other potentials (and IAS15) that need GSL splines or other
sources that are not built here.  This script links once with
``--no-undefined`` to learn which symbols the linker cannot resolve, writes a
stub for each (it prints a message and aborts if ever called; the potentials
integrated here never reach one), and links again.

Usage: python ref_stubs.py <out.so> <obj>... -- <link flags>
"""
import os
import re
import subprocess
import sys


def main(argv):
    out = argv[1]
    sep = argv.index("--")
    objs = argv[2:sep]
    flags = argv[sep + 1 :]
    cc = os.environ.get("ORACLE_CC", "/usr/bin/gcc")
    cmd = [cc, "-shared", "-o", out, *objs, "-Wl,--no-undefined", *flags]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    names = sorted(set(re.findall(r"undefined reference to `([^']+)'", proc.stderr)))
    stub_c = os.path.join(os.path.dirname(out), "stubs.c")
    with open(stub_c, "w") as f:
        f.write("/* generated by oracle/ref_stubs.py: unresolved reference symbols */\n")
        f.write("#include <stdio.h>\n#include <stdlib.h>\n")
        f.write("static void ref_stub_hit(const char *n)\n{ fprintf(stderr, \"oracle/_ref: %s is not built\\n\", n); abort(); }\n")
        for n in names:
            f.write(f"void {n}(void) {{ ref_stub_hit(\"{n}\"); }}\n")
    stub_o = stub_c[:-2] + ".o"
    subprocess.run([cc, "-O2", "-fPIC", "-c", stub_c, "-o", stub_o], check=True)
    subprocess.run([cc, "-shared", "-o", out, *objs, stub_o, "-Wl,--no-undefined", *flags], check=True)
    print(f"linked {out} with {len(names)} stubs")


if __name__ == "__main__":
    main(sys.argv)
