"""Builds tests/golden/libgen_inputs.so from gen_inputs.cpp (g++, no other dependency)."""
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SO = HERE / "libgen_inputs.so"


def build(force: bool = False) -> Path:
    src = HERE / "gen_inputs.cpp"
    if force or not SO.exists() or SO.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", str(SO), str(src)],
                       check=True)
    return SO


if __name__ == "__main__":
    print(build(force=True))
