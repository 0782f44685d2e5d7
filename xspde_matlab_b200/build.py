"""Build libxspde_b200.so in-tree (host C++ + embedded sm_100a kernel sources).

The problem kernels are generated per problem and compiled at run time by
NVRTC for sm_100a; their hand-written source lives in csrc/kernels/*.cuh and
is embedded into the library here.  The AOT translation units are compiled by
nvcc with -gencode arch=compute_100a,code=sm_100a.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libxspde_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
KERNELS = [("prelude", "xs_prelude.cuh"), ("noise", "xs_noise.cuh"), ("resident", "xs_resident.cuh"),
           ("stream_common", "xs_stream_common.cuh"), ("stream", "xs_stream.cuh"), ("stream3", "xs_stream3.cuh"),
           ("stream3_tc", "xs_stream3_tc.cuh")]
SOURCES = ["xs_capi.cpp", "xs_expr.cpp", "xs_aot.cu", "xs_noalloc.cu", "xs_mlp.cu"]


def _embed():
    out = os.path.join(CSRC, "_kernel_sources.cpp")
    parts = ["// generated by build.py from csrc/kernels/*.cuh -- do not edit\n"]
    for name, fn in KERNELS:
        with open(os.path.join(CSRC, "kernels", fn)) as f:
            text = f.read()
        assert ")XSRC\"" not in text
        parts.append('extern const char* xs_kernel_source_%s;\nconst char* xs_kernel_source_%s = R"XSRC(%s)XSRC";\n'
                     % (name, name, text))
    data = "".join(parts)
    if not os.path.exists(out) or open(out).read() != data:
        with open(out, "w") as f:
            f.write(data)
    return out


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(CSRC, "xs_expr.hpp"),
                                                      os.path.join(CSRC, "xs_noalloc.hpp"),
                                                      os.path.join(CSRC, "xs_mlp.hpp"),
                                                      os.path.join(HERE, "build.py"),
                                                      os.path.join(os.path.dirname(HERE), "include", "xspde_b200.h")]
    deps += [os.path.join(CSRC, "kernels", k) for _, k in KERNELS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    emb = _embed()
    if not force and not _stale():
        return LIB
    nvcc = os.path.join(CUDA, "bin", "nvcc")
    inc = os.path.join(os.path.dirname(HERE), "include")
    cmd = [nvcc, "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
           "-I", inc, "-I", CSRC, "-o", LIB + ".tmp"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES] + [emb]
    cmd += ["-L", os.path.join(CUDA, "lib64"), "-lnvrtc", "-cudart", "static", "-ldl", "-lrt", "-lpthread",
            "-Xlinker", "-rpath," + os.path.join(CUDA, "lib64")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
