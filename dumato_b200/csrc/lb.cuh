// Device-side warp-level load balancing: a root cursor, a lock-free donation queue and
// termination detection, all inside one persistent kernel.
//
// This replaces the reference's host-mediated "stop the world" balancing
// (src/main/DuMatoCPU.cu:386-562: poll d_status every 100 ms, raise d_stop, copy every
// warp's stack to the host, donate (prefix, last extension) jobs from the heaviest warps
// to idle ones, copy back, relaunch). Here a task is (root, item range): the items of a
// root are the units its DFS is split into (local edges for cliques, second vertices for
// motifs). A warp that finds the root cursor exhausted announces itself hungry; a busy
// warp whose task has run for a while and sees hungry warps splits its remaining item
// range in half and enqueues the upper half (a donated DFS prefix). The receiver rebuilds
// the root's state and runs only the donated items.
//
// The queue is a set of bounded multi-producer multi-consumer rings (per-slot sequence
// numbers): a consumer only ever takes a slot whose producer has finished writing it, so
// nothing waits on another warp's store. Donations are demand-limited: a warp donates only
// while more warps are hungry than tasks are queued. Termination: `pending` counts roots not yet finished plus
// donated tasks not yet finished (raised before the enqueue). A hungry warp leaves when
// pending is zero; if nothing changes for timeout_ns it records ERR_TIMEOUT and leaves.
//
// Every hot word lives on its own 128-byte line so that polling hungry warps and busy
// warps do not queue behind each other at one L2 slice.
#pragma once

#include <cstdint>

#include "engine.hpp"

namespace dmb {

// A queued task. level 0: items [begin, end) of root's first level. level L >= 1 (motifs):
// positions [begin, end) of the extension set at DFS level L, reached from the root along
// path[0] (the second vertex's index in E_0) and path[1..L-1] (the chosen index at each
// level below L) - a donated DFS prefix.
constexpr int QPATH = 7;
struct QSlot {
  unsigned seq;
  int root;
  int begin;
  int end;
  int level;
  int path[QPATH];
  int pad[4];
};

// Persistent queue: nq shard headers followed by nq x cap slots (shard s owns slots
// [s*cap, (s+1)*cap)). Positions keep running across calls (a call ends with the queue
// empty); the host re-initialises it after an error. A warp pushes to and pops from its home
// shard first and then the others, so thousands of hungry warps do not all contend on one
// read position.
struct QHeader {
  unsigned write_pos;
  unsigned pad0[31];
  unsigned read_pos;
  unsigned pad1[31];
};

struct LBArgs {
  DevCounters* ctr;
  QHeader* qh;                // nq shard headers
  QSlot* q;                   // nq * qcap slots
  int qcap;                   // slots per shard
  int hungry_trigger;    // donate when at least this many warps are hungry (<= 0: never)
  int max_donations;     // per task
  long long donate_after_ns;  // a task donates only after running this long
  long long timeout_ns;
  int test_stall;             // test hook: wait at exit on a word nothing sets
  int min_split;              // a task keeps ranges shorter than this
  int nq;                     // shards
};

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int vload(const int* p) { return *reinterpret_cast<const volatile int*>(p); }
__device__ __forceinline__ unsigned vloadu(const unsigned* p) { return *reinterpret_cast<const volatile unsigned*>(p); }
__device__ __forceinline__ unsigned long long vload64(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}

__device__ __forceinline__ void set_err(DevCounters* c, int code) { atomicCAS(&c->err, 0, code); }

static __device__ __forceinline__ bool shard_push(const LBArgs& lb, int sh, int root, int b, int e, int level,
                                                  const int* path) {
  QHeader* h = lb.qh + sh;
  QSlot* base = lb.q + (size_t)sh * lb.qcap;
  unsigned pos = vloadu(&h->write_pos);
  for (int tries = 0; tries < 64; ++tries) {
    QSlot* s = base + (pos % (unsigned)lb.qcap);
    const unsigned seq = vloadu(&s->seq);
    const int dif = (int)(seq - pos);
    if (dif == 0) {
      const unsigned prev = atomicCAS(&h->write_pos, pos, pos + 1);
      if (prev == pos) {
        s->root = root;
        s->begin = b;
        s->end = e;
        s->level = level;
        for (int i = 0; i < level && i < QPATH; ++i) s->path[i] = path[i];
        __threadfence();
        atomicExch(&s->seq, pos + 1);
        return true;
      }
      pos = prev;
    } else if (dif < 0) {
      return false;  // this shard is full
    } else {
      pos = vloadu(&h->write_pos);
    }
  }
  return false;
}

static __device__ __forceinline__ bool shard_pop(const LBArgs& lb, int sh, int& root, int& b, int& e, int& level,
                                                 int* path) {
  QHeader* h = lb.qh + sh;
  QSlot* base = lb.q + (size_t)sh * lb.qcap;
  unsigned pos = vloadu(&h->read_pos);
  for (int tries = 0; tries < 64; ++tries) {
    QSlot* s = base + (pos % (unsigned)lb.qcap);
    const unsigned seq = vloadu(&s->seq);
    const int dif = (int)(seq - (pos + 1));
    if (dif == 0) {
      const unsigned prev = atomicCAS(&h->read_pos, pos, pos + 1);
      if (prev == pos) {
        __threadfence();
        const volatile QSlot* vs = s;
        root = vs->root;
        b = vs->begin;
        e = vs->end;
        level = vs->level;
        for (int i = 0; i < level && i < QPATH; ++i) path[i] = vs->path[i];
        __threadfence();
        atomicExch(&s->seq, pos + (unsigned)lb.qcap);
        return true;
      }
      pos = prev;
    } else if (dif < 0) {
      return false;  // empty (or a producer is still writing its slot)
    } else {
      pos = vloadu(&h->read_pos);
    }
  }
  return false;
}

static __device__ __noinline__ bool q_push(const LBArgs& lb, int home, int root, int b, int e, int level,
                                           const int* path) {
  for (int i = 0; i < lb.nq; ++i)
    if (shard_push(lb, (home + i) % lb.nq, root, b, e, level, path)) {
      atomicAdd(&lb.ctr->queued, 1);
      return true;
    }
  return false;
}

static __device__ __noinline__ bool q_pop(const LBArgs& lb, int home, int& root, int& b, int& e, int& level,
                                          int* path) {
  if (vload(&lb.ctr->queued) <= 0) return false;
  for (int i = 0; i < lb.nq; ++i)
    if (shard_pop(lb, (home + i) % lb.nq, root, b, e, level, path)) {
      atomicSub(&lb.ctr->queued, 1);
      return true;
    }
  return false;
}

// Lane-0 only. Claims a chunk of roots [first, first+count) from the cursor, or failing
// that a donated task (count = 1, range [b, e)). Returns false when all work is done or an
// error was raised. A caller that defers the pending-count decrements of the roots it has
// finished passes their number in *unflushed: they are subtracted before the caller waits
// for work (so `pending` can reach zero), and *unflushed is reset.
// A caller that passes `idle` (polls, waiting ns) gets its waiting statistics added there
// instead of to the global counters, to be summed per block at exit.
static __device__ __noinline__ bool lb_next(const LBArgs& lb, int n_roots, int total_warps, int& first, int& count,
                                            int& b, int& e, bool& donated, int& level, int* path,
                                            int* unflushed = nullptr, unsigned long long* idle = nullptr) {
  DevCounters* c = lb.ctr;
  int cur = vload(&c->cursor);
  if (cur < n_roots) {
    // light tail roots are claimed several at a time to keep the cursor line cool
    int chunk = (n_roots - cur) / (8 * total_warps);
    chunk = chunk < 1 ? 1 : (chunk > 16 ? 16 : chunk);
    const int r = atomicAdd(&c->cursor, chunk);
    if (r < n_roots) {
      first = r;
      count = min(chunk, n_roots - r);
      b = 0;
      e = -1;
      level = 0;
      donated = false;
      return true;
    }
  }
  if (unflushed && *unflushed) {
    __threadfence();
    atomicSub(&c->pending, *unflushed);
    *unflushed = 0;
  }
  atomicAdd(&c->hungry, 1);
  const long long t_hungry = global_ns();
  long long t0 = t_hungry;
  unsigned long long last = vload64(&c->progress);
  int last_pending = vload(&c->pending);
  unsigned backoff = 128;
  unsigned long long polls = 0;
  bool got = false;
  const int home = (int)((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) % (unsigned)lb.nq);
  while (true) {
    int root = 0;
    if (q_pop(lb, home, root, b, e, level, path)) {
      first = root;
      count = 1;
      donated = true;
      got = true;
      break;
    }
    const int pend = vload(&c->pending);
    if (pend <= 0 && lb.test_stall) {
      // test hook: wait for test_gate, which nothing sets, until the bounded wait gives up
      const long long ts = global_ns();
      while (vload(&c->test_gate) == 0) {
        if (global_ns() - ts > lb.timeout_ns) {
          set_err(c, ERR_TIMEOUT);
          break;
        }
        __nanosleep(2000);
      }
      break;
    }
    if (pend <= 0 || vload(&c->err) != 0) break;
    const unsigned long long p = vload64(&c->progress);
    if (p != last || pend != last_pending) {
      last = p;
      last_pending = pend;
      t0 = global_ns();
    } else if (global_ns() - t0 > lb.timeout_ns) {
      set_err(c, ERR_TIMEOUT);
      break;
    }
    ++polls;
    __nanosleep(backoff);
    // the back-off cap grows with the time spent waiting: short kernels see their end
    // within about a microsecond, long waits poll the shared words at most every 16 us
    const long long waited = global_ns() - t_hungry;
    const unsigned cap = waited < 250000 ? 1024u : 16384u;
    backoff = backoff < cap ? backoff << 1 : cap;
  }
  // a warp that leaves because all work is done need not withdraw its demand
  if (got || !idle) atomicSub(&c->hungry, 1);
  const unsigned long long waited_ns = (unsigned long long)(global_ns() - t_hungry);
  if (idle) {
    idle[0] += polls;
    idle[1] += waited_ns;
  } else {
    if (polls) atomicAdd(&c->idle_polls, polls);
    atomicAdd(&c->hungry_ns, waited_ns);
  }
  return got;
}

// Records a finished task's duration (lane 0).
__device__ __forceinline__ void lb_task_time(const LBArgs& lb, long long t_start, int root) {
  const unsigned long long dur = (unsigned long long)(global_ns() - t_start);
  const unsigned long long old = atomicMax(&lb.ctr->max_task_ns, dur);
  if (dur > old) lb.ctr->max_task_root = root;
}

__device__ __forceinline__ void lb_done(const LBArgs& lb, int count) {
  __threadfence();
  atomicSub(&lb.ctr->pending, count);
}

// Item range of a task over n items. Donated ranges are [b, e) (e < 0: to the end). A root
// pre-split by the scheduler into P parts is encoded b = -1 - p, e = -1 - P and covers
// [p*n/P, (p+1)*n/P); whole roots come as (0, -1).
__device__ __forceinline__ void task_range(int b, int e, int n, int& lo, int& hi) {
  if (b < 0) {
    const int p = -1 - b, P = -1 - e;
    lo = (int)((long long)p * n / P);
    hi = (int)((long long)(p + 1) * n / P);
  } else {
    lo = b;
    hi = e < 0 ? n : min(e, n);
  }
}

// Decodes a scheduler part word into (b, e).
__device__ __forceinline__ void part_bounds(int part, int& b, int& e) {
  const int pp = part & ~PART_EAGER;
  if (pp) {
    b = -1 - (pp & 0xffff);
    e = -1 - ((pp >> 16) & 0x3fff);
  }
}

// Item range of the running task, packed as (next | end << 32) in shared memory. Taking an
// item is one 64-bit atomicAdd (the low word is the cursor; it only ever passes `end` by
// the number of lanes that find the range empty); splitting off a donation is one CAS.
__device__ __forceinline__ unsigned long long pack_range(int next, int end) {
  return (unsigned long long)(unsigned)next | ((unsigned long long)(unsigned)end << 32);
}

__device__ __forceinline__ int range_take(unsigned long long* range) {
  const unsigned long long old = atomicAdd(range, 1ull);
  const int next = (int)(unsigned)old, end = (int)(unsigned)(old >> 32);
  return next < end ? next : -1;
}

// Split point of items [next, end) (at least two): the midpoint, or with cost_tail > 0 (item
// i costs about cost_tail - i) the point where the remaining cost halves.
__device__ __forceinline__ int split_mid(int next, int end, int cost_tail) {
  if (cost_tail <= 0) return next + (end - next + 1) / 2;
  const double a = (double)(cost_tail - next) + 0.5;
  const double total = 0.5 * (double)(end - next) * (double)((cost_tail - next) + (cost_tail - end + 1));
  const double disc = a * a - total;
  const int x = (int)(a - sqrt(disc > 0 ? disc : 0.0) + 0.5);
  return next + max(1, min(end - next - 1, x));
}

// Splits the upper part of the remaining items [next, end) of a task's range off and
// enqueues it as (root, [mid, end)) at `level` with `path` (with cost_tail > 0, item i is
// taken to cost cost_tail - i and the split halves the remaining cost instead of the item
// count; a range is split only with at least min_items (default lb.min_split) left). Returns
// true when the queue was full: the split-off items [ob, oe) then belong to the caller, who
// must run them itself (lanes that find the range empty have already moved the cursor past
// `mid`, so the split cannot simply be undone). `busy` serialises donations of one warp.
__device__ __forceinline__ bool range_split_donate(const LBArgs& lb, unsigned long long* range, int root,
                                                   int* donations_left, int* busy, int& ob, int& oe, int cost_tail,
                                                   int min_items, int level, const int* path, bool* donated = nullptr) {
  if (*reinterpret_cast<volatile int*>(donations_left) <= 0) return false;
  if (atomicCAS(busy, 0, 1) != 0) return false;
  bool own = false;
  unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(range);
  while (true) {
    const int next = (int)(unsigned)cur, end = (int)(unsigned)(cur >> 32);
    const int need = min_items > 0 ? min_items : lb.min_split;
    if (end - next < (need > 2 ? need : 2)) break;
    const int mid = split_mid(next, end, cost_tail);
    const unsigned long long prev = atomicCAS(range, cur, pack_range(next, mid));
    if (prev != cur) {
      cur = prev;
      continue;
    }
    atomicAdd(&lb.ctr->pending, 1);
    const int home = (int)((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) % (unsigned)lb.nq);
    if (q_push(lb, home, root, mid, end, level, path)) {
      atomicSub(donations_left, 1);
      atomicAdd(&lb.ctr->donations, 1ull);
      if (level > 0) atomicAdd(&lb.ctr->prefix_donations, 1ull);
      if (donated) *donated = true;
    } else {
      atomicSub(&lb.ctr->pending, 1);
      ob = mid;
      oe = end;
      own = true;
    }
    break;
  }
  atomicExch(busy, 0);
  return own;
}

// If more warps are hungry than tasks are queued and the task has run longer than
// donate_after_ns (or `eager`), splits the range as range_split_donate does.
__device__ __forceinline__ bool range_maybe_donate(const LBArgs& lb, unsigned long long* range, int root,
                                                   int* donations_left, long long task_start, int* busy, int& ob,
                                                   int& oe, int cost_tail = 0, int min_items = 0, int level = 0,
                                                   const int* path = nullptr, bool eager = false) {
  if (lb.hungry_trigger <= 0) return false;
  if (*reinterpret_cast<volatile int*>(donations_left) <= 0) return false;
  // demand: hungry warps not yet served by a queued task
  const int hungry = vload(&lb.ctr->hungry);
  if (hungry - vload(&lb.ctr->queued) < lb.hungry_trigger) return false;
  if (!eager && global_ns() - task_start < lb.donate_after_ns) return false;
  return range_split_donate(lb, range, root, donations_left, busy, ob, oe, cost_tail, min_items, level, path);
}

// Demand test shared by the donation paths (lane 0): hungry warps outnumber queued tasks by
// the trigger and the task has run long enough.
__device__ __forceinline__ bool lb_wants_donation(const LBArgs& lb, const int* donations_left, long long task_start) {
  if (lb.hungry_trigger <= 0) return false;
  if (*reinterpret_cast<const volatile int*>(donations_left) <= 0) return false;
  if (vload(&lb.ctr->hungry) - vload(&lb.ctr->queued) < lb.hungry_trigger) return false;
  return global_ns() - task_start >= lb.donate_after_ns;
}

// Enqueues a deep task (lane 0). Returns false when every shard is full.
__device__ __forceinline__ bool lb_donate_deep(const LBArgs& lb, int root, int level, const int* path, int b, int e) {
  atomicAdd(&lb.ctr->pending, 1);
  const int home = (int)((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) % (unsigned)lb.nq);
  if (q_push(lb, home, root, b, e, level, path)) {
    atomicAdd(&lb.ctr->donations, 1ull);
    if (level > 0) atomicAdd(&lb.ctr->prefix_donations, 1ull);
    return true;
  }
  atomicSub(&lb.ctr->pending, 1);
  return false;
}

}  // namespace dmb
