// tb_batch.cpp -- caller-side batching of block contractions.
//
// TAVP-WRK executes the block contractions of a tensor instruction one
// talsh_tensor_contract at a time (INTERVIRT/tavp_worker.F90:9420-9518, call
// at :9467), each a separate launch sequence.  A batch collects such calls
// (same pattern, data kind, alpha and accumulation) and runs them at flush
// time as one grouped tensor-core launch (tb_bsc_plan_create +
// tb_bsc_execute).  Iterative methods issue the same block list again and
// again, so every flushed list is remembered with its plan: a list equal to
// an earlier one (same tasks in the same order) replays that plan's CUDA
// graph, and on its second use the plan's tile and slice choice is timed
// once (tb_bsc_autotune, which leaves D unchanged).  Data kinds the grouped
// kernel does not take (complex) run as a loop of tb_tensor_contract_str
// calls on the same stream, with the same accumulation rule: the flag
// applies to each output block once per flush.
#include <cstdint>
#include <cstring>
#include <list>
#include <string>
#include <unordered_set>
#include <vector>

#include "talsh_b200.h"
#include "tb_pattern.h"

namespace {

constexpr size_t kMaxCachedPlans = 8;
constexpr int kR4 = 4, kR8 = 8;  // TAL-SH data kinds the grouped kernel takes

struct CachedPlan {
  std::string key;   // the task list's bytes
  tb_bsc_plan_t* plan = nullptr;
  int uses = 0;
};

}  // namespace

struct tb_batch_s {
  std::string pattern;
  int dtk = 0;
  double ar = 1.0, ai = 0.0;
  int accumulative = 1;
  tb_plan_t plan{};
  bool has_plan = false;
  std::vector<tb_block_task_t> queue;
  std::list<CachedPlan> cache;  // most recently used first
  tb_batch_stats_t stats{};
};

using tb::set_error;

extern "C" int tb_batch_create(const char* pattern, int data_kind, double alpha_real, double alpha_imag,
                               int accumulative, const tb_plan_t* plan, tb_batch_t** out) {
  if (!pattern || !out) { set_error("tb_batch_create: bad arguments"); return TB_ERR_INVALID_ARGS; }
  *out = nullptr;
  tb::ParsedPattern P;
  if (tb::parse_pattern(pattern, &P) || P.rrank < 0) {
    set_error("tb_batch_create: not a contraction pattern: %s", pattern);
    return TB_ERR_INVALID_ARGS;
  }
  if (tb_data_kind_size(data_kind) <= 0) { set_error("tb_batch_create: bad data kind %d", data_kind); return TB_ERR_INVALID_ARGS; }
  tb_batch_t* b = new tb_batch_t;
  b->pattern = pattern;
  b->dtk = data_kind;
  b->ar = alpha_real;
  b->ai = alpha_imag;
  b->accumulative = accumulative ? 1 : 0;
  if (plan) { b->plan = *plan; b->has_plan = true; }
  *out = b;
  return 0;
}

extern "C" int tb_batch_add(tb_batch_t* b, int n, const tb_block_task_t* tasks) {
  if (!b || n < 0 || (n > 0 && !tasks)) { set_error("tb_batch_add: bad arguments"); return TB_ERR_INVALID_ARGS; }
  b->queue.insert(b->queue.end(), tasks, tasks + n);
  return 0;
}

extern "C" int tb_batch_pending(const tb_batch_t* b) { return b ? (int)b->queue.size() : -1; }

namespace {

int run_loop(tb_batch_t* b, void* stream) {
  tb::ParsedPattern P;
  tb::parse_pattern(b->pattern.c_str(), &P);
  std::unordered_set<const void*> seen;
  for (const tb_block_task_t& t : b->queue) {
    const int acc = seen.insert(t.d).second ? b->accumulative : 1;
    if (int e = tb_tensor_contract_str(b->pattern.c_str(), b->dtk, P.drank, t.d_dims, t.d, P.lrank, t.l_dims, t.l,
                                       P.rrank, t.r_dims, t.r, b->ar, b->ai, acc, b->has_plan ? &b->plan : nullptr,
                                       stream))
      return e;
  }
  b->stats.loop_flushes++;
  return 0;
}

}  // namespace

extern "C" int tb_batch_flush(tb_batch_t* b, void* stream) {
  if (!b) { set_error("tb_batch_flush: null batch"); return TB_ERR_INVALID_ARGS; }
  if (b->queue.empty()) return 0;
  int err = 0;
  if (b->dtk != kR8 && b->dtk != kR4) {
    err = run_loop(b, stream);
  } else {
    std::string key((const char*)b->queue.data(), b->queue.size() * sizeof(tb_block_task_t));
    auto it = b->cache.begin();
    for (; it != b->cache.end(); ++it)
      if (it->key == key) break;
    if (it != b->cache.end()) {
      b->cache.splice(b->cache.begin(), b->cache, it);  // most recently used first
      b->stats.plan_reuses++;
    } else {
      tb_bsc_plan_t* pl = nullptr;
      err = tb_bsc_plan_create(b->pattern.c_str(), b->dtk, (int)b->queue.size(), b->queue.data(), b->ar, b->ai,
                               b->accumulative, b->has_plan ? &b->plan : nullptr, &pl, stream);
      if (err == TB_ERR_NOT_IMPLEMENTED) {
        pl = nullptr;
        err = run_loop(b, stream);  // a pattern the grouped kernel does not take
      } else if (!err) {
        b->stats.plans_built++;
        if (b->cache.size() >= kMaxCachedPlans) {
          tb_bsc_plan_destroy(b->cache.back().plan);
          b->cache.pop_back();
        }
        b->cache.push_front(CachedPlan{std::move(key), pl, 0});
      }
      if (!pl) {
        if (!err) b->stats.tasks += (int64_t)b->queue.size();
        b->queue.clear();
        return err;
      }
    }
    CachedPlan& c = b->cache.front();
    if (++c.uses == 2) {
      if ((err = tb_bsc_autotune(c.plan, stream))) { b->queue.clear(); return err; }
      b->stats.autotunes++;
    }
    err = tb_bsc_execute(c.plan, stream);
    b->stats.grouped_flushes++;
  }
  b->stats.tasks += (int64_t)b->queue.size();
  b->queue.clear();
  return err;
}

extern "C" int tb_batch_get_stats(const tb_batch_t* b, tb_batch_stats_t* st) {
  if (!b || !st) { set_error("tb_batch_get_stats: bad arguments"); return TB_ERR_INVALID_ARGS; }
  *st = b->stats;
  st->cached_plans = (int)b->cache.size();
  return 0;
}

extern "C" int tb_batch_destroy(tb_batch_t* b) {
  if (!b) return 0;
  for (auto& c : b->cache) tb_bsc_plan_destroy(c.plan);
  delete b;
  return 0;
}
