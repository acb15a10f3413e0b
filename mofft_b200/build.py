"""Build libmofft.so (C host library + sm_100a kernels) and the oracle.

Steps:
  1. regenerate the radix codelets and the wisdom table (mofft_b200/codegen);
  2. compute the build ID: sha256 over every source that goes into the
     library (the B200 analogue of the reference's content-derived
     MOFFT_BINARY_ID, CMakeLists.txt:51-93);
  3. compile the CUDA translation units with nvcc for sm_100a and the C host
     units with gcc, in parallel, into mofft_b200/_build/;
  4. link mofft_b200/lib/libmofft.so (static CUDA runtime) and
     oracle/liboracle.so.

Run:  python -m mofft_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libmofft.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources() -> tuple[list[Path], list[Path], list[Path]]:
    cu = sorted(CSRC.glob("*.cu"))
    c = sorted(CSRC.glob("*.c"))
    headers = sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) +
                     list((CSRC / "generated").glob("*")) +
                     list((ROOT / "include").glob("*.h")))
    return cu, c, headers


def build_id(files: list[Path]) -> str:
    digest = hashlib.sha256()
    for path in sorted(files):
        digest.update(path.relative_to(ROOT).as_posix().encode())
        digest.update(b"\0")
        digest.update(path.read_bytes())
        digest.update(b"\0")
    return digest.hexdigest()


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stdout}")


def _stale(obj: Path, deps: list[Path], stamp: str) -> bool:
    tag = obj.with_suffix(obj.suffix + ".id")
    if not obj.exists() or not tag.exists() or tag.read_text() != stamp:
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def generate() -> None:
    from mofft_b200.codegen import compile_wisdom, gen_codelets
    gen_codelets.main(["gen", str(CSRC / "generated")])
    compile_wisdom.main(["wisdom"])


def public_symbols() -> list[str]:
    """Every function declared in include/*.h: the only symbols libmofft.so
    exports (a linker version script hides the internal ones)."""
    import re
    names = set()
    for header in sorted((ROOT / "include").glob("*.h")):
        for match in re.finditer(r"\b(mofft_[a-z0-9_]+)\s*\(", header.read_text()):
            names.add(match.group(1))
    return sorted(names)


def build_library(force: bool = False, jobs: int | None = None) -> Path:
    generate()
    cu, c, headers = _sources()
    bid = build_id(cu + c + headers)
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    common_defs = [f'-DMOFFT_BINARY_ID="{bid}"']
    jobs_list = []
    objs = []
    for src in cu:
        obj = BUILD / (src.stem + ".cu.o")
        objs.append(obj)
        # only the build ID definition differs between builds; kernels do not
        # depend on it, so .cu objects are keyed on their own sources
        if force or _stale(obj, [src] + headers, "cu"):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
            jobs_list.append((obj, "cu", cmd))
    for src in c:
        obj = BUILD / (src.stem + ".c.o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers, bid):
            cmd = ["gcc", "-O2", "-g", "-fPIC", "-std=gnu11", "-Wall", "-Wextra",
                   "-Wno-unused-parameter", "-I", str(CSRC), "-I", str(CUDA_HOME / "include"),
                   *common_defs, "-c", str(src), "-o", str(obj)]
            jobs_list.append((obj, bid, cmd))
    if jobs_list:
        workers = jobs or min(len(jobs_list), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=workers) as pool:
            futures = {pool.submit(_run, cmd): (obj, stamp) for obj, stamp, cmd in jobs_list}
            for fut in cf.as_completed(futures):
                fut.result()
                obj, stamp = futures[fut]
                obj.with_suffix(obj.suffix + ".id").write_text(stamp)
    script = BUILD / "exports.map"
    text = "{\n  global:\n" + "".join(f"    {n};\n" for n in public_symbols()) + \
        "  local: *;\n};\n"
    if not script.exists() or script.read_text() != text:
        script.write_text(text)
        force = True
    if force or jobs_list or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp),
              *[str(o) for o in objs], f"-Xlinker=--version-script={script}",
              "-lpthread", "-lm", "-ldl", "-lrt"])
        os.replace(tmp, LIB)
    (PKG / "lib" / "BUILD_ID").write_text(bid + "\n")
    return LIB


def build_oracle(force: bool = False) -> Path:
    srcs = sorted(ORACLE_DIR.glob("*.c"))
    hdrs = sorted(ORACLE_DIR.glob("*.h"))
    if not srcs:
        raise RuntimeError("oracle sources missing")
    newest = max(p.stat().st_mtime for p in srcs + hdrs)
    if force or not ORACLE_LIB.exists() or ORACLE_LIB.stat().st_mtime < newest:
        tmp = ORACLE_LIB.with_suffix(".so.tmp")
        _run(["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared",
              "-std=gnu11", "-Wall", "-o", str(tmp), *[str(s) for s in srcs], "-lm"])
        os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def main(argv: list[str]) -> int:
    force = "--force" in argv
    if not shutil.which(NVCC) and not Path(NVCC).exists():
        print("nvcc not found", file=sys.stderr)
        return 1
    lib = build_library(force)
    print(f"built {lib}")
    print(f"built {build_oracle(force)}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
