"""Build libgpawfd.so (the sm_100a CUDA library) in-tree with nvcc.

    python -m gpaw_b200.build            # incremental
    python -m gpaw_b200.build --force    # rebuild everything

Each .cu in csrc/ compiles to an object under _build/ in parallel; the
objects link into gpaw_b200/libgpawfd.so with the CUDA runtime linked
statically, so the library does not depend on which libcudart the host
process (for example PyTorch) loaded.
"""
import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
INCLUDE = os.path.join(ROOT, 'include')
LIB = os.path.join(HERE, 'libgpawfd.so')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ['-O3', '-std=c++17', '-lineinfo', '--expt-relaxed-constexpr',
              '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden',
              '-I' + INCLUDE, '-I' + CSRC]


def nvcc():
    path = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(path):
        raise RuntimeError('nvcc not found')
    return path


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith('.cu'))


def _local_includes(path, seen):
    """Headers of this package that `path` includes, transitively."""
    for line in open(path):
        m = re.match(r'\s*#\s*include\s+"([^"]+)"', line)
        if not m:
            continue
        for d in (CSRC, INCLUDE):
            h = os.path.join(d, m.group(1))
            if os.path.exists(h) and h not in seen:
                seen.add(h)
                _local_includes(h, seen)
                break
    return seen


def _compile(src, force, ptxas_verbose):
    obj = os.path.join(BUILD, src[:-3] + '.o')
    srcp = os.path.join(CSRC, src)
    deps = [srcp] + sorted(_local_includes(srcp, set()))
    if (not force and os.path.exists(obj) and
            os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps)):
        return obj, ''
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ['-c', srcp, '-o', obj]
    if ptxas_verbose:
        cmd += ['-Xptxas', '-v']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('nvcc failed for %s:\n%s%s' % (src, r.stdout, r.stderr))
    return obj, r.stderr


def build(force=False, ptxas_verbose=False, jobs=None, quiet=True):
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, force, ptxas_verbose), srcs))
    objs = [o for o, _ in results]
    if ptxas_verbose:
        for _, log in results:
            sys.stderr.write(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ['-shared', '-cudart', 'static', '-o', LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError('link failed:\n%s%s' % (r.stdout, r.stderr))
    if not quiet:
        print('built', LIB)
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--ptxas', action='store_true', help='print -Xptxas -v resource usage')
    a = ap.parse_args()
    build(force=a.force, ptxas_verbose=a.ptxas, quiet=False)
