"""Build recipe for libterrain_b200.so (sm_100a) and its test-only host twin.

  python build.py            generate evaluators from model/ and compile lib/libterrain_b200.so
  python build.py --host     also compile lib/libterrain_b200_hostcheck.so: the same
                             per-element bodies built for the host CPU, used only by the
                             CPU test suite to check the generated code against the oracle

Exactness flags: device code -fmad=false -prec-div=true -prec-sqrt=true -ftz=false
(no fast math); host code -ffp-contract=off.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
GEN = os.path.join(HERE, '_gen')
LIB = os.path.join(HERE, 'lib')
MODEL = os.path.join(HERE, 'model')
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')

DEVICE_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-std=c++17', '-lineinfo', '-fmad=false', '-prec-div=true',
                '-prec-sqrt=true', '-ftz=false']
HOST_FLAGS = ['-Xcompiler', '-fPIC,-ffp-contract=off,-O2,-fno-fast-math']
if os.environ.get('TB_PTXAS_VERBOSE'):
    DEVICE_FLAGS.append('-Xptxas=-v')


def run(cmd):
    print(' '.join(cmd), flush=True)
    subprocess.check_call(cmd)


TUNING = os.path.join(HERE, 'tuning', 'launch_table.txt')


def generate():
    sys.path.insert(0, os.path.join(HERE, 'codegen'))
    import gen_eval
    r = gen_eval.generate(os.path.join(MODEL, 'overworld_ir.json'), os.path.join(MODEL, 'overworld_terrain.json'),
                          os.path.join(GEN, 'model_gen.cuh'))
    write_launch_table()
    return r


def write_launch_table():
    """_gen/launch_table.h: the committed launch table as a string constant (parsed by the
    library at tg_create); rewritten only when its contents change."""
    with open(TUNING) as f:
        text = f.read()
    body = '// generated by build.py from tuning/launch_table.txt\n#pragma once\nnamespace tb {\nstatic const char kLaunchTableText[] =\n'
    body += ''.join('    "%s\\n"\n' % line.replace('\\', '\\\\').replace('"', '\\"') for line in text.splitlines())
    body += '    "";\n}  // namespace tb\n'
    out = os.path.join(GEN, 'launch_table.h')
    if not os.path.exists(out) or open(out).read() != body:
        os.makedirs(GEN, exist_ok=True)
        with open(out, 'w') as f:
            f.write(body)


def newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(GEN, 'model_gen.cuh'), os.path.join(GEN, 'launch_table.h')]


def build_device(force=False, out=None, defines=()):
    os.makedirs(LIB, exist_ok=True)
    out = out or os.path.join(LIB, 'libterrain_b200.so')
    if not force and not newer(out, sources()):
        return out
    objs = []
    tag = os.path.splitext(os.path.basename(out))[0]
    for src in ('terrain.cu', 'tb_host.cpp'):
        obj = os.path.join(os.path.dirname(out), '%s.%s.o' % (tag, src))
        run([NVCC] + DEVICE_FLAGS + HOST_FLAGS + ['-D%s' % d for d in defines] + ['-I', CSRC, '-I', GEN, '-c', os.path.join(CSRC, src), '-o', obj])
        objs.append(obj)
    run([NVCC, '-shared', '-gencode', 'arch=compute_100a,code=sm_100a', '-o', out] + objs + ['-lcudart'])
    return out


def build_host(force=False):
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, 'libterrain_b200_hostcheck.so')
    deps = sources() + [os.path.join(HERE, '..', 'tests', 'hostcheck', 'hostcheck.cpp')]
    if not force and not newer(out, deps):
        return out
    run(['g++', '-std=c++17', '-O2', '-ffp-contract=off', '-fno-fast-math', '-fPIC', '-shared', '-DTB_COUNT_OPS', '-I', CSRC, '-I', GEN,
         os.path.join(HERE, '..', 'tests', 'hostcheck', 'hostcheck.cpp'), os.path.join(CSRC, 'tb_host.cpp'), '-o', out])
    return out


def main(argv):
    generate()
    force = '--force' in argv
    build_device(force)
    if '--host' in argv:
        build_host(force)


if __name__ == '__main__':
    main(sys.argv[1:])
