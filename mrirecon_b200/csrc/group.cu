// Recorder of grouped launches (group.cuh) and its C entry points.
//
// mrb_group_begin(n) opens a recording for n problems; mrb_group_select(i)
// directs the following entry-point calls to problem i; their kernel
// launches are stored, not issued.  mrb_group_end(stream) issues them on one
// stream: each step takes the body that is next in the most problems' record
// lists (ties: the lowest problem index first), launches the next record of
// every problem whose next record runs that body as one grouped launch (a
// plain launch when only one problem has it) and advances those problems.
// Every problem's own records therefore run in the order it made them, each
// after all of its earlier ones, and different problems never share data.
#include <mutex>
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

int flush(Recorder& R, cudaStream_t st) {
  const int n = (int)R.lists.size();
  std::vector<size_t> head(n, 0);
  std::vector<const LaunchRec*> batch;
  batch.reserve(n);
  long long nrec = 0, nlaunch = 0;
  auto same = [](const LaunchRec& a, const LaunchRec& b) { return a.key == b.key && a.threads == b.threads; };
  for (;;) {
    // the body that is next in the most lists
    const LaunchRec* best = nullptr;
    int best_count = 0;
    for (int i = 0; i < n; ++i) {
      if (head[i] >= R.lists[i].size()) continue;
      const LaunchRec& ri = R.lists[i][head[i]];
      int c = 0;
      for (int j = 0; j < n; ++j)
        if (head[j] < R.lists[j].size() && same(R.lists[j][head[j]], ri)) ++c;
      if (c > best_count) {
        best_count = c;
        best = &ri;
      }
    }
    if (best == nullptr) break;
    const LaunchRec& b = *best;
    batch.clear();
    for (int j = 0; j < n; ++j) {
      if (head[j] >= R.lists[j].size()) continue;
      const LaunchRec& rj = R.lists[j][head[j]];
      if (!same(rj, b)) continue;
      batch.push_back(&rj);
      ++head[j];
    }
    nrec += (long long)batch.size();
    const int rc = batch.size() == 1 ? b.single(*batch[0], st) : b.group(batch.data(), (int)batch.size(), st);
    if (rc) return rc;
    ++nlaunch;
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
  R.lists[R.cur].push_back(std::move(r));
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
