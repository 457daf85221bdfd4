// Recorder of grouped launches (group.cuh) and its C entry points.
//
// mrb_group_begin(n) opens a recording for n problems; mrb_group_select(i)
// directs the following entry-point calls to problem i; their kernel
// launches are stored, not issued.  mrb_group_end(stream) issues them on
// `stream` in steps.  A step is a (kernel step, occurrence) pair: the k-th
// record of step "fwd_rows" of every problem belongs to the same replay step,
// whatever the FFT length of each problem.  Steps are ordered consistently
// with every problem's own record order (a topological order of the steps,
// earliest first); the records of a step that run the same body form one
// grouped launch, and when one step needs launches of several bodies, all but
// the first run on auxiliary streams forked from `stream` and joined back
// before the next step, so they overlap.  Every problem's records therefore
// run in the order it made them, each after all of its earlier ones, and
// different problems never share data.  Records without a kernel step (none
// of the library's grouped bodies lacks one) each form a step of their own.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <queue>
#include <set>
#include <tuple>
#include <vector>

#include "group.cuh"

namespace mrb {

namespace {

struct Recorder {
  bool active = false;
  int cur = 0;
  std::vector<std::vector<LaunchRec>> lists;
  long long last_records = 0, last_launches = 0;
};

Recorder& rec() {
  static Recorder r;
  return r;
}

std::mutex g_group_mu;   // one recording at a time per process

// auxiliary streams and events of one device, created on first use
struct Aux {
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
};

int aux_for(int n, Aux** out) {
  static std::map<int, Aux> per_dev;
  int dev = 0;
  MRB_CUDA_TRY(cudaGetDevice(&dev));
  Aux& a = per_dev[dev];
  if (!a.fork) MRB_CUDA_TRY(cudaEventCreateWithFlags(&a.fork, cudaEventDisableTiming));
  while ((int)a.streams.size() < n) {
    cudaStream_t s = nullptr;
    cudaEvent_t e = nullptr;
    MRB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    MRB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    a.streams.push_back(s);
    a.joins.push_back(e);
  }
  *out = &a;
  return 0;
}

bool same_step(const LaunchRec& a, const LaunchRec& b) {
  if (a.family == nullptr || b.family == nullptr) return false;
  return a.occ == b.occ && std::strcmp(a.family, b.family) == 0;
}

bool same_body(const LaunchRec& a, const LaunchRec& b) { return a.key == b.key && a.threads == b.threads; }

int launch_batch(const std::vector<const LaunchRec*>& b, cudaStream_t st) {
  return b.size() == 1 ? b[0]->single(*b[0], st) : b[0]->group(b.data(), (int)b.size(), st);
}

int flush(Recorder& R, cudaStream_t st) {
  const int n = (int)R.lists.size();
  // steps: one per distinct (family, occurrence); a record without a family is a step of its own
  std::vector<std::vector<int>> step_of(n);
  std::vector<const LaunchRec*> step_rep;        // a representative record
  std::vector<std::vector<std::pair<int, int>>> members;   // (problem, index)
  std::vector<size_t> first_pos;                  // earliest position at which the step occurs
  for (int i = 0; i < n; ++i) {
    step_of[i].resize(R.lists[i].size());
    for (size_t j = 0; j < R.lists[i].size(); ++j) {
      const LaunchRec& r = R.lists[i][j];
      int s = -1;
      for (int k = 0; k < (int)step_rep.size() && r.family; ++k)
        if (same_step(*step_rep[k], r)) {
          s = k;
          break;
        }
      if (s < 0) {
        s = (int)step_rep.size();
        step_rep.push_back(&r);
        members.emplace_back();
        first_pos.push_back(j);
      }
      step_of[i][j] = s;
      members[s].emplace_back(i, (int)j);
      first_pos[s] = std::min(first_pos[s], j);
    }
  }
  const int ns = (int)step_rep.size();
  // order constraints from every problem's consecutive records
  std::vector<std::set<int>> succ(ns);
  std::vector<int> indeg(ns, 0);
  for (int i = 0; i < n; ++i)
    for (size_t j = 1; j < step_of[i].size(); ++j) {
      const int a = step_of[i][j - 1], b = step_of[i][j];
      if (a != b && succ[a].insert(b).second) ++indeg[b];
    }
  using Item = std::tuple<size_t, int>;   // (earliest position, step)
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> ready;
  for (int s = 0; s < ns; ++s)
    if (indeg[s] == 0) ready.emplace(first_pos[s], s);
  std::vector<int> order;
  order.reserve(ns);
  while (!ready.empty()) {
    const int s = std::get<1>(ready.top());
    ready.pop();
    order.push_back(s);
    for (int t : succ[s])
      if (--indeg[t] == 0) ready.emplace(first_pos[t], t);
  }
  // a step that repeats within one problem, or problems that order two steps
  // differently, leave a cycle: issue every problem's records on its own then
  bool ok = (int)order.size() == ns;
  for (int s = 0; ok && s < ns; ++s) {
    std::set<int> seen;
    for (auto& m : members[s]) ok = ok && seen.insert(m.first).second;
  }
  long long nrec = 0, nlaunch = 0;
  if (!ok) {
    for (int i = 0; i < n; ++i)
      for (const LaunchRec& r : R.lists[i]) {
        if (int rc = r.single(r, st)) return rc;
        ++nrec;
        ++nlaunch;
      }
    R.last_records = nrec;
    R.last_launches = nlaunch;
    return 0;
  }
  for (int s : order) {
    // the step's records, grouped by body in problem order
    std::vector<std::vector<const LaunchRec*>> bodies;
    for (auto& m : members[s]) {
      const LaunchRec* r = &R.lists[m.first][m.second];
      auto it = std::find_if(bodies.begin(), bodies.end(), [&](const std::vector<const LaunchRec*>& b) {
        return same_body(*b[0], *r);
      });
      if (it == bodies.end()) bodies.push_back({r});
      else it->push_back(r);
    }
    nrec += (long long)members[s].size();
    nlaunch += (long long)bodies.size();
    if (bodies.size() == 1) {
      if (int rc = launch_batch(bodies[0], st)) return rc;
      continue;
    }
    Aux* aux = nullptr;
    if (int rc = aux_for((int)bodies.size() - 1, &aux)) return rc;
    MRB_CUDA_TRY(cudaEventRecord(aux->fork, st));
    for (size_t b = 1; b < bodies.size(); ++b) {
      cudaStream_t as = aux->streams[b - 1];
      MRB_CUDA_TRY(cudaStreamWaitEvent(as, aux->fork, 0));
      if (int rc = launch_batch(bodies[b], as)) return rc;
      MRB_CUDA_TRY(cudaEventRecord(aux->joins[b - 1], as));
    }
    if (int rc = launch_batch(bodies[0], st)) return rc;
    for (size_t b = 1; b < bodies.size(); ++b) MRB_CUDA_TRY(cudaStreamWaitEvent(st, aux->joins[b - 1], 0));
  }
  R.last_records = nrec;
  R.last_launches = nlaunch;
  return 0;
}

}  // namespace

bool group_recording() { return rec().active; }

int group_record(LaunchRec&& r) {
  Recorder& R = rec();
  if (R.cur < 0 || R.cur >= (int)R.lists.size()) return fail(MRB_ESTATE, "no problem selected in the recording");
  std::vector<LaunchRec>& l = R.lists[R.cur];
  r.occ = 0;
  if (r.family)
    for (const LaunchRec& q : l)
      if (q.family && std::strcmp(q.family, r.family) == 0) ++r.occ;
  l.push_back(std::move(r));
  return 0;
}

int set_max_smem(const void* fn, size_t bytes, size_t* done) {
  if (bytes <= 48 * 1024 || bytes <= *done) return 0;
  MRB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  *done = bytes;
  return 0;
}

}  // namespace mrb

extern "C" int mrb_group_begin(int nproblems) {
  MRB_REQUIRE(nproblems >= 1 && nproblems <= 4096, "nproblems must be in [1, 4096] (got %d)", nproblems);
  std::lock_guard<std::mutex> lk(mrb::g_group_mu);
  mrb::Recorder& R = mrb::rec();
  if (R.active) return mrb::fail(MRB_ESTATE, "a recording is already open");
  R.lists.assign(nproblems, {});
  R.cur = 0;
  R.active = true;
  return 0;
}

extern "C" int mrb_group_select(int problem) {
  mrb::Recorder& R = mrb::rec();
  if (!R.active) return mrb::fail(MRB_ESTATE, "no recording is open");
  MRB_REQUIRE(problem >= 0 && problem < (int)R.lists.size(), "problem %d outside [0, %d)", problem,
              (int)R.lists.size());
  R.cur = problem;
  return 0;
}

extern "C" int mrb_group_end(mrb_stream_t stream) {
  std::lock_guard<std::mutex> lk(mrb::g_group_mu);
  mrb::Recorder& R = mrb::rec();
  if (!R.active) return mrb::fail(MRB_ESTATE, "no recording is open");
  R.active = false;   // the replay launches for real
  const int rc = mrb::flush(R, (cudaStream_t)stream);
  R.lists.clear();
  return rc;
}

extern "C" int mrb_group_cancel(void) {
  std::lock_guard<std::mutex> lk(mrb::g_group_mu);
  mrb::Recorder& R = mrb::rec();
  R.active = false;
  R.lists.clear();
  return 0;
}

extern "C" int mrb_group_stats(int64_t* records, int64_t* launches) {
  MRB_REQUIRE(records != nullptr && launches != nullptr, "null output");
  *records = mrb::rec().last_records;
  *launches = mrb::rec().last_launches;
  return 0;
}
