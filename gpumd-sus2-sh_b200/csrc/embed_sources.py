"""Build step: writes a C++ include holding the device headers of the per-edge
kernels as raw string literals, so the library can compile any model shape
with NVRTC at load time (edge_jit.cpp).

    python3 embed_sources.py OUT.inc HEADER...
"""
import os
import sys

DELIM = "sus2jit"


def main() -> None:
    out, headers = sys.argv[1], sys.argv[2:]
    names, bodies = [], []
    for h in headers:
        with open(h) as fh:
            text = fh.read()
        if ")" + DELIM + '"' in text:
            raise SystemExit(f"{h} contains the raw-string delimiter")
        names.append(os.path.basename(h))
        bodies.append(text)
    with open(out + ".tmp", "w") as fh:
        fh.write("// generated by embed_sources.py; do not edit\n")
        fh.write(f"static const int kJitHeaderCount = {len(names)};\n")
        fh.write("static const char* const kJitHeaderNames[] = {"
                 + ", ".join(f'"{n}"' for n in names) + "};\n")
        fh.write("static const char* const kJitHeaderSources[] = {\n")
        for b in bodies:
            fh.write(f'R"{DELIM}({b}){DELIM}",\n')
        fh.write("};\n")
    os.replace(out + ".tmp", out)


if __name__ == "__main__":
    main()
