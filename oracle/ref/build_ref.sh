#!/usr/bin/env bash
# Build recipe for the reference-backed oracle binaries (test infrastructure only).
#
# The reference (XKRT) targets clang >= 20; this image has g++ 13 only. g++ rejects four
# clang-isms, so this script makes a PATCHED COPY of the reference's header tree under
# oracle/_ref/include (git-ignored build output, never committed) and compiles our own
# harness sources (oracle/ref/*.cc) against it plus a handful of the reference's .cc files
# read in place. The reference tree itself is never modified.
#
#   P1 include/xkrt/memory/access/common/khp-tree.hpp: in-class explicit specialisations of
#      `includes_t<S,H>` -> partial specialisations over an extra defaulted parameter.
#   P2 blas/dependency-tree.hpp, blas/memory-tree.hpp: constructors spelled `Node<K>(` -> `Node(`.
#   P3 task/task.hpp: `void (*F)(Args..., task_t *)` is non-deducible in g++ -> generic `FN F`.
#   P4 thread/thread.h: non-template `commit` overloads for the two callback shapes used.
#   flags: -std=c++20 (c++23 for the runtime sources, whose <stdatomic.h> needs it in g++ 13)
#          -D_Static_assert=static_assert -include list -DNDEBUG
#   generated: support.h (CMake defaults, every vendor driver off), version.h, an hwloc shim.
#
# Usage: oracle/ref/build_ref.sh REFERENCE_ROOT   (or XK_REFERENCE_ROOT in the environment)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REPO="$(cd "$HERE/../.." && pwd)"
REF="${1:-${XK_REFERENCE_ROOT:-}}"
OUT="$REPO/oracle/_ref"
if [ -z "$REF" ]; then
    echo "usage: $0 REFERENCE_ROOT (or set XK_REFERENCE_ROOT)" >&2
    exit 2
fi

if [ ! -d "$REF/include/xkrt" ]; then
    echo "build_ref.sh: reference tree not found at $REF; skipping (prebuilt binaries, if any, are kept)" >&2
    exit 0
fi

mkdir -p "$OUT"
rm -rf "$OUT/include" "$OUT/shim"
mkdir -p "$OUT/include" "$OUT/shim/hwloc"
cp -r "$REF/include/xkrt" "$OUT/include/xkrt"
chmod -R u+w "$OUT/include"
INC="$OUT/include/xkrt"

# ---- P1: includes_t specialisations -------------------------------------------------------
python3 - "$INC/memory/access/common/khp-tree.hpp" <<'PY'
import re, sys
p = sys.argv[1]
s = open(p).read()
s = s.replace("template <bool S, bool H>\n                struct includes_t {};",
              "template <bool S, bool H, typename D = void>\n                struct includes_t {};", 1)
n = 0
for a, b in (("true", "true"), ("true", "false"), ("false", "true"), ("false", "false")):
    old = "template<>\n                struct includes_t<%s, %s> {" % (a, b)
    new = "template<typename D>\n                struct includes_t<%s, %s, D> {" % (a, b)
    if old in s:
        s = s.replace(old, new, 1); n += 1
if n != 4:
    sys.exit("P1: expected 4 specialisations, patched %d" % n)
open(p, "w").write(s)
PY

# ---- P2: template-id constructors ---------------------------------------------------------
sed -i 's/^\(\s*\)KBLASDependencyTreeNode<K>(/\1KBLASDependencyTreeNode(/' "$INC/memory/access/blas/dependency-tree.hpp"
sed -i 's/^\(\s*\)KBLASMemoryTreeNode<K>(/\1KBLASMemoryTreeNode(/' "$INC/memory/access/blas/memory-tree.hpp"

# ---- P3: non-deducible callback parameter packs --------------------------------------------
python3 - "$INC/task/task.hpp" <<'PY'
import sys
p = sys.argv[1]
s = open(p).read()
old = "template <typename... Args>\nstatic inline void\n%s(\n%s    void (*F)(Args..., task_t *),"
cnt = 0
for fn, pre in (("__task_ready", "    task_t * task,\n"),
                ("__task_commit", "    task_t * task,\n"),
                ("__task_fetched", "    task_wait_counter_type_t n,\n    task_t * task,\n")):
    o = old % (fn, pre)
    n = "template <typename FN, typename... Args>\nstatic inline void\n%s(\n%s    FN F," % (fn, pre)
    if o in s:
        s = s.replace(o, n, 1); cnt += 1
if cnt != 3:
    sys.exit("P3: expected 3 callback signatures, patched %d" % cnt)
open(p, "w").write(s)
PY

# ---- P4: commit overloads -------------------------------------------------------------------
python3 - "$INC/thread/thread.h" <<'PY'
import sys
p = sys.argv[1]
s = open(p).read()
anchor = "        template <typename... Args>\n        inline void\n        commit(\n"
if anchor not in s:
    sys.exit("P4: commit template not found")
extra = (
"        inline void commit(task_t * task, void (*F)(struct runtime_t *, task_t *), struct runtime_t * r)\n"
"        { assert(this->current_task); ++this->current_task->cc; task->parent = this->current_task;"
" __task_commit(task, F, r); }\n"
"        inline void commit(task_t * task, void (*F)(struct runtime_t *, struct team_t *, task_t *), struct runtime_t * r, struct team_t * t)\n"
"        { assert(this->current_task); ++this->current_task->cc; task->parent = this->current_task;"
" __task_commit(task, F, r, t); }\n\n")
s = s.replace(anchor, extra + anchor, 1)
open(p, "w").write(s)
PY

# ---- generated headers ---------------------------------------------------------------------
sed -e 's/@USE_MEMORY_REGISTER_OVERFLOW_PROTECTION@/1/' \
    -e 's/@USE_MEMORY_REGISTER_PAGE@/1/' \
    -e 's/@USE_MEMORY_REGISTER_ASSISTED@/1/' \
    -e 's/@[A-Z_]*@/0/g' \
    "$REF/include/xkrt/support.h.in" > "$INC/support.h"
sed -e 's/£GIT_HASH/reference-oracle/' "$REF/include/xkrt/version.template" > "$INC/version.h"

# ---- hwloc shim: thread placement only; every call is a no-op -------------------------------
cat > "$OUT/shim/hwloc.h" <<'H'
#ifndef XK_HWLOC_SHIM_H
#define XK_HWLOC_SHIM_H
#include <sched.h>
typedef struct hwloc_topology_s * hwloc_topology_t;
typedef struct hwloc_bitmap_s { int dummy; } * hwloc_bitmap_t;
typedef hwloc_bitmap_t hwloc_cpuset_t;
typedef const struct hwloc_bitmap_s * hwloc_const_cpuset_t;
typedef enum { HWLOC_OBJ_MACHINE, HWLOC_OBJ_PACKAGE, HWLOC_OBJ_CORE, HWLOC_OBJ_PU, HWLOC_OBJ_L1CACHE,
               HWLOC_OBJ_L2CACHE, HWLOC_OBJ_L3CACHE, HWLOC_OBJ_NUMANODE } hwloc_obj_type_t;
typedef struct hwloc_obj { hwloc_cpuset_t cpuset; unsigned logical_index; unsigned os_index; char * name; } * hwloc_obj_t;
static inline int hwloc_topology_init(hwloc_topology_t * t) { *t = 0; return 0; }
static inline int hwloc_topology_load(hwloc_topology_t) { return 0; }
static inline void hwloc_topology_destroy(hwloc_topology_t) {}
static inline int hwloc_get_type_depth(hwloc_topology_t, hwloc_obj_type_t) { return 0; }
static inline int hwloc_get_nbobjs_by_depth(hwloc_topology_t, int) { return 1; }
static inline int hwloc_get_nbobjs_by_type(hwloc_topology_t, hwloc_obj_type_t) { return 1; }
static inline hwloc_obj_t hwloc_get_obj_by_type(hwloc_topology_t, hwloc_obj_type_t, unsigned) { return 0; }
static inline hwloc_obj_t hwloc_get_obj_by_depth(hwloc_topology_t, int, unsigned) { return 0; }
static inline hwloc_bitmap_t hwloc_bitmap_alloc(void) { return 0; }
static inline void hwloc_bitmap_free(hwloc_bitmap_t) {}
#endif
H
cat > "$OUT/shim/hwloc/glibc-sched.h" <<'H'
#ifndef XK_HWLOC_GLIBC_SHIM_H
#define XK_HWLOC_GLIBC_SHIM_H
#include <hwloc.h>
static inline int hwloc_cpuset_to_glibc_sched_affinity(hwloc_topology_t, hwloc_const_cpuset_t,
                                                       cpu_set_t * s, size_t) { CPU_ZERO(s); return 0; }
#endif
H

CXX="${XK_ORACLE_CXX:-g++}"   # the g++ on PATH (g++ 13.3); a CXX from the environment may lack C++23 <stdatomic.h>
CXXFLAGS="-std=c++20 -O2 -DNDEBUG -D_Static_assert=static_assert -include list -w -I$OUT/include -I$OUT/shim -I$REF/api/c/include"

# ---- transfer-plan oracle: reference memory tree under the canonical schedule ----------------
"$CXX" $CXXFLAGS -include array -o "$OUT/ref_plan" \
    "$HERE/ref_plan.cc" "$HERE/seams.cc" "$REF/src/task/task.cc" "$REF/src/logger/logger.cc" -lpthread
echo "built $OUT/ref_plan"

# ---- host-only runtime (CPU baseline): the reference's runtime sources + its host driver ------
OBJ="$OUT/obj"
mkdir -p "$OBJ"
RT_SRCS="src/memory/access.cc src/conf/conf.cc src/debug/cairo.cc src/distribution/distribution.cc src/driver.cc
 src/driver/device.cc src/driver/driver.cc src/driver/queue.cc src/driver/driver_host.cc src/file/readwrite.cc
 src/logger/logger.cc src/logger/metric.cc src/memory.cc src/memory/coherent.cc src/memory/copy.cc
 src/memory/distribute.cc src/memory/invalidate.cc src/memory/register.cc src/power.cc src/runtime.cc src/sched.cc
 src/stats/stats.cc src/task.cc src/task/format.cc src/task/task.cc src/thread/deque.cc src/thread/thread.cc"
OBJS=""
for s in $RT_SRCS; do
    o="$OBJ/$(echo "$s" | tr '/' '_').o"
    "$CXX" ${CXXFLAGS/-std=c++20/-std=c++23} -c "$REF/$s" -o "$o" &
    OBJS="$OBJS $o"
done
wait
# ---- dependency oracle: reference trees driven by src/task/task.cc; the runtime's thread
# sources give the handle map's extra tasks their task stack (thread_t::get_tls)
"$CXX" ${CXXFLAGS/-std=c++20/-std=c++23} -o "$OUT/ref_deps" "$HERE/ref_deps.cc" $OBJS -lpthread -ldl
echo "built $OUT/ref_deps"
"$CXX" ${CXXFLAGS/-std=c++20/-std=c++23} -o "$OUT/ref_heat" "$HERE/ref_heat.cc" $OBJS -lpthread -ldl
echo "built $OUT/ref_heat"
"$CXX" ${CXXFLAGS/-std=c++20/-std=c++23} -o "$OUT/ref_axpby" "$HERE/ref_axpby.cc" $OBJS -lpthread -ldl
echo "built $OUT/ref_axpby"
