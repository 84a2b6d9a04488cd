"""Build the reference's own CUDA implementation (DTmaxwell4) for sm_100a
into oracle/_ref/ -- test infrastructure only, the independent check of the
engine and of the CPU oracle.

The reference keeps its stencil kernels in a Python-2 generator
(genDT.py + genAlg.py, Makefile:157-158) and builds one executable with
compile-time sizes (-DNS -DNP -DNA -DNV, Makefile:57-59).  This recipe

  1. copies the reference's sources from the reference tree into
     oracle/_ref/<variant>/src (so the tree itself is never written);
  2. sets NDev to 1 in the copy of py_consts.h (the reference splits y into
     stripes over two GPUs, py_consts.h:15, params.h:66-90; one GPU here);
  3. replaces im2D.h with the headless stand-in of stubs/im2D.h (GLUT and PNG,
     not used by _main --test) and force-includes stubs/legacy_tex.h
     (CUDA 12 removed texture references; the Maxwell kernels do not read
     them, COFFS_IN_DEVICE);
  4. converts the generator to Python 3 (py2to3.py), runs genDT.py, and checks
     that both iteration orders of the dict loop the conversion had to touch
     generate identical kernels;
  5. compiles the reference's translation units as its Makefile lists them
     (dt.o from DTmxw.cu, texmodel.o, ker{D,S,Is,Id,Xs,Xd}[_pmls].o,
     ker[I]TFSF[_pmls].o; -rdc, -O3, OpenMP) for sm_100a with the reference's
     DROP_DATA switch on (field drops after every big step), plus
     stubs/im3D_stubs.cu (the visualiser's symbols) and ref_run.cpp (the
     run.py driver), and links oracle/_ref/<variant>/ref_run.

The reference's own build system is not run; its sources are compiled as they
are, apart from the NDev setting above.

Usage: python oracle/refbuild/build_ref.py [--np 60 --na 60 --nv 128 --ns 20] [--double] [--jobs 8]
"""
import argparse
import concurrent.futures as cf
import filecmp
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT_ROOT = os.path.join(ORACLE, "_ref")
DEFAULT_REF = "/root/reference"

SOURCES = ["DTmxw.cu", "diamond.cu", "drop.cu", "texmodel.cu", "texmodel.cuh", "copyrags.cuh", "chooseV.h",
           "cuda_math.h", "cuda_math_double.h", "defs.h", "params.h", "py_consts.h", "init.h", "signal.h",
           "signal.hpp", "lambda_func.hpp", "sensor.h", "window.hpp", "dispersion.cpp", "im3D.hpp",
           "Arr3Dpars.hpp", "genAlg.py", "genDT.py"]
# Makefile:127-135 (AsyncTYPES) and :116-123
KERNELS = ["D_pmls", "S_pmls", "Is_pmls", "Id_pmls", "Xs_pmls", "Xd_pmls", "D", "S", "Is", "Id", "Xs", "Xd",
           "TFSF", "TFSF_pmls", "ITFSF", "ITFSF_pmls"]


def variant_name(a):
    return "np%d_na%d_nv%d_ns%d%s" % (a.np, a.na, a.nv, a.ns, "_f64" if a.double else "")


def binary_path(np_=60, na=60, nv=128, ns=20, double=False):
    """Path of the ref_run executable of one size variant (may not exist)."""
    a = argparse.Namespace(np=np_, na=na, nv=nv, ns=ns, double=double)
    return os.path.join(OUT_ROOT, variant_name(a), "ref_run")


def run(cmd, cwd, env=None):
    res = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, env=env)
    if res.returncode != 0:
        raise RuntimeError("command failed (%s):\n%s\n%s%s" % (cwd, " ".join(cmd), res.stdout[-4000:], res.stderr[-8000:]))
    return res


def prepare_sources(ref, src):
    if os.path.isdir(src):
        shutil.rmtree(src)
    os.makedirs(src)
    for f in SOURCES:
        shutil.copy(os.path.join(ref, f), os.path.join(src, f))
    consts = os.path.join(src, "py_consts.h")
    text = open(consts).read()
    if text.count("#define NDev 2") != 1:
        raise RuntimeError("py_consts.h: expected one '#define NDev 2'")
    open(consts, "w").write(text.replace("#define NDev 2", "#define NDev 1"))
    shutil.copy(os.path.join(HERE, "stubs", "im2D.h"), os.path.join(src, "im2D.h"))
    for f in ("genAlg.py", "genDT.py"):
        run([sys.executable, os.path.join(HERE, "py2to3.py"), os.path.join(ref, f), os.path.join(src, f)], src)


def generate(src):
    env = dict(os.environ, PYTHONWARNINGS="ignore")
    run([sys.executable, "genDT.py"], src, env)
    check = os.path.join(src, "_order_check")
    os.makedirs(check)
    for f in ("genAlg.py", "genDT.py"):
        shutil.copy(os.path.join(src, f), check)
    run([sys.executable, "genDT.py"], check, dict(env, REFGEN_ORDER="reversed"))
    gen = sorted(f for f in os.listdir(src) if f.endswith(".inc.cu"))
    if len(gen) != 50:
        raise RuntimeError("generator produced %d files, expected 50" % len(gen))
    for f in gen:
        if not filecmp.cmp(os.path.join(src, f), os.path.join(check, f), shallow=False):
            raise RuntimeError("generated %s depends on the dict iteration order" % f)
    shutil.rmtree(check)


def build(ref=DEFAULT_REF, np_=60, na=60, nv=128, ns=20, double=False, jobs=8, force=False, verbose=False):
    a = argparse.Namespace(np=np_, na=na, nv=nv, ns=ns, double=double)
    out = os.path.join(OUT_ROOT, variant_name(a))
    exe = os.path.join(out, "ref_run")
    if not os.path.isdir(ref):
        raise RuntimeError("reference sources not found at %s" % ref)
    recipe = [os.path.join(HERE, f) for f in ("ref_run.cpp", "py2to3.py", "build_ref.py")]
    recipe += [os.path.join(HERE, "stubs", f) for f in os.listdir(os.path.join(HERE, "stubs"))]
    newest = max(os.path.getmtime(f) for f in recipe)
    if os.path.exists(exe) and not force and os.path.getmtime(exe) >= newest:
        return exe
    src, obj = os.path.join(out, "src"), os.path.join(out, "obj")
    if force and os.path.isdir(obj):
        shutil.rmtree(obj)
    os.makedirs(obj, exist_ok=True)
    if force or not os.path.exists(os.path.join(src, "kerD.inc.cu")):
        prepare_sources(ref, src)
        generate(src)
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    # DROP_DATA is the reference's own switch (py_consts.h:18): calcStep then writes ragEz_<step>.arr,
    # Ez of one node per rag over the whole domain, after every big step (diamond.cu:487-489, drop.cu:83-107)
    defs = ["-DNS=%d" % ns, "-DNP=%d" % np_, "-DNA=%d" % na, "-DNV=%d" % nv, "-DDROP_DATA"] + (["-DUSE_DOUBLE"] if double else [])
    gencode = ["-gencode", "arch=compute_100a,code=sm_100a"]
    common = [nvcc, "-O3", "-rdc=true", "-std=c++14", "-w", "-I", src, "-include", os.path.join(HERE, "stubs", "legacy_tex.h"),
              "--compiler-options=-O3 -fopenmp -fPIC -w -fpermissive"] + gencode + defs
    # DTmxw.cu's own main() (DTmxw.cu:835) is renamed: ref_run.cpp is the program's main, as run.py is
    units = [("dt.o", os.path.join(src, "DTmxw.cu"), ["-Dmain=reference_standalone_main"]),
             ("texmodel.o", os.path.join(src, "texmodel.cu"), []),
             ("im3D_stubs.o", os.path.join(HERE, "stubs", "im3D_stubs.cu"), [])]
    units += [("ker%s.o" % k, os.path.join(src, "ker%s.inc.cu" % k), ["-x", "cu"]) for k in KERNELS]

    def compile_unit(u):
        o, s, extra = u
        deps = [s, os.path.join(HERE, "stubs", "legacy_tex.h"), os.path.join(HERE, "stubs", "im2D.h")]
        if os.path.exists(os.path.join(obj, o)) and os.path.getmtime(os.path.join(obj, o)) >= max(map(os.path.getmtime, deps)):
            return o
        res = run(common + ["-Xptxas", "-v"] + extra + ["-c", s, "-o", os.path.join(obj, o)], src)
        with open(os.path.join(obj, o + ".log"), "w") as f:
            f.write(res.stderr)
        return o

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for o in ex.map(compile_unit, units):
            if verbose:
                print("compiled", o, flush=True)
    drv = os.path.join(obj, "ref_run.o")
    run([nvcc, "-O2", "-std=c++14", "-w", "-I", src] + defs + ["-x", "c++", "-c", os.path.join(HERE, "ref_run.cpp"), "-o", drv], src)
    objs = [os.path.join(obj, u[0]) for u in units] + [drv]
    run([nvcc, "-rdc=true"] + gencode + objs + ["-o", exe + ".tmp", "-lgomp", "-lpthread"], out)
    os.replace(exe + ".tmp", exe)
    return exe


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--ref", default=DEFAULT_REF)
    p.add_argument("--np", type=int, default=60)
    p.add_argument("--na", type=int, default=60)
    p.add_argument("--nv", type=int, default=128)
    p.add_argument("--ns", type=int, default=20)
    p.add_argument("--double", action="store_true")
    p.add_argument("--jobs", type=int, default=8)
    p.add_argument("--force", action="store_true")
    a = p.parse_args()
    print(build(a.ref, a.np, a.na, a.nv, a.ns, a.double, a.jobs, a.force, verbose=True))


if __name__ == "__main__":
    main()
