// fc_batch.cu -- the batched form: many periodic boxes, each taken through
// mass assignment, the periodic CLI normalisation and the periodic
// correlator, captured once into a single CUDA graph and replayed.
//
// Per box (one lane stream of the graph):
//   memset grid -> K-key -> radix sort -> K-tiles -> K-scatter colour passes
//   (fc_assign.cu) -> k_norm_pad: (rho - mean) / mean into the FP32 or FP64
//   padded work grid (fftcorr.cc:369-375 fused with array_ops.cc:35-53) ->
//   r2c -> |F|^2 -> k-subgrids per ell -> c2r -> r-subgrids per ell
//   (correlator.h:273-357, fc_corr.cu)
// and after all lanes join, one persistent chunk-reduction kernel and one
// fold kernel produce every histogram of every box (the same sums, in the
// same order, as the per-box BinIndex::reduce).
//
// Boxes are spread over the lanes by a greedy longest-first balance of their
// estimated cost.  The launch shapes of the grid-stride kernels, the lane
// count and the histogram kernel's CTA count come from the autotuner table
// (timed on first use, or imported).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "fc_internal.h"

namespace fc {
namespace {

// add_scalar(-mean) then multiply_by(1/mean) (fftcorr.cc:369-375), written
// straight into the padded work grid in the transform precision.  mean =
// totw / ncells from the assignor's device totals.
template <typename TI, typename T>
__global__ void k_norm_pad(const TI *__restrict__ rho, T *__restrict__ work,
                           int n0, int n1, int n2, int n2p,
                           const double *__restrict__ totals, double ncells) {
  const double mean = totals[0] / ncells;
  const double shift = -mean;
  const double scale = 1.0 / mean;
  const size_t nrows = (size_t)n0 * n1;
  for (size_t row = blockIdx.x; row < nrows; row += gridDim.x) {
    const TI *src = rho + row * n2;
    T *dst = work + row * n2p;
    // Rounded to the cell type after each step, as fc_grid_add_scalar and
    // fc_grid_multiply_by round a grid's cells (a no-op for FP64 cells).
    for (int k = threadIdx.x; k < n2; k += blockDim.x)
      dst[k] = (T)((double)(TI)((double)src[k] + shift) * scale);
  }
}

// Persistent chunk reductions over the work items of every box: item i is
// summed exactly as k_chunk_sums sums chunk i of one BinIndex.
__global__ void __launch_bounds__(kHistThreads)
    k_batch_chunks(const HistItem *__restrict__ items, int n,
                   double *__restrict__ partials) {
  __shared__ double red[32];
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const HistItem h = items[it];
    double acc = 0.0;
    for (int i = threadIdx.x; i < h.len; i += blockDim.x)
      acc += h.values[h.perm[h.start + i]];
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) partials[it] = acc;
  }
}

// One thread per bin of every box: its chunk partials folded in order.
__global__ void k_batch_fold(const FoldItem *__restrict__ folds, int n,
                             const double *__restrict__ partials) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const FoldItem f = folds[i];
    double s = 0.0;
    for (int c = f.first; c < f.first + f.count; ++c) s += partials[c];
    *f.dest = s;
  }
}

}  // namespace

// ------------------------------------------------------------ autotuner
// Process-wide table of tuned launch parameters, keyed by kernel, precision
// and problem size ("abs2 f32 384x384x384").  Values are two integers whose
// meaning depends on the kernel (threads and waves for grid-stride kernels,
// the lane count, the histogram kernel's CTA count).
namespace tune {
std::mutex mu;
std::map<std::string, std::pair<int, int>> &table() {
  static std::map<std::string, std::pair<int, int>> t;
  return t;
}
bool get(const std::string &k, std::pair<int, int> *v) {
  std::lock_guard<std::mutex> g(mu);
  auto it = table().find(k);
  if (it == table().end()) return false;
  *v = it->second;
  return true;
}
void put(const std::string &k, std::pair<int, int> v) {
  std::lock_guard<std::mutex> g(mu);
  table()[k] = v;
}
std::string shape_key(const char *kernel, bool fp64, const int s[3]) {
  char buf[96];
  std::snprintf(buf, sizeof(buf), "%s %s %dx%dx%d", kernel, fp64 ? "f64" : "f32",
                s[0], s[1], s[2]);
  return buf;
}
}  // namespace tune

namespace {

// Times f() (which enqueues on s) with events: one warm-up, then the
// minimum of `reps` single runs, in milliseconds.
template <typename F>
float time_on(cudaStream_t s, F f, int reps = 3) {
  cudaEvent_t a, b;
  FC_CUDA(cudaEventCreate(&a));
  FC_CUDA(cudaEventCreate(&b));
  f();
  float best = 1e30f;
  for (int r = 0; r < reps; ++r) {
    FC_CUDA(cudaEventRecord(a, s));
    f();
    FC_CUDA(cudaEventRecord(b, s));
    FC_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    FC_CUDA(cudaEventElapsedTime(&ms, a, b));
    best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

const int kThreadChoices[] = {128, 256, 512};
const int kWaveChoices[] = {2, 4, 8, 16, 32};

}  // namespace

struct BatchBox {
  int shape[3];
  double cell;
  const double *posw;
  int64_t n;
};

struct Batch {
  fc_batch_params prm;
  std::vector<BatchBox> boxes;
  std::vector<std::unique_ptr<Grid>> grids;
  std::vector<Assignor *> mas;
  std::vector<Correlator *> corrs;
  std::vector<LaunchShape> ls_norm;
  std::vector<int> lane_of;
  int nlanes = 0;
  int hist_blocks = 0;
  std::vector<cudaStream_t> lanes;
  cudaStream_t main = nullptr;
  cudaEvent_t fork_ev = nullptr, t0 = nullptr, t1 = nullptr;
  std::vector<cudaEvent_t> join_ev;
  std::vector<HistItem> items;
  std::vector<FoldItem> folds;
  DeviceBuffer d_items, d_folds, d_partials;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t graph_nodes = 0, kernel_nodes = 0;
  unsigned long long own_kernels = 0;
  size_t device_bytes = 0;
  double last_seconds = 0.0;

  bool fp64() const { return prm.precision == FC_FP64; }

  explicit Batch(const fc_batch_params &p) : prm(p) {}

  // Builds everything; on failure the destructor releases what was built.
  void init(const fc_batch_box *bx, int nboxes) {
    FC_REQUIRE(nboxes > 0, FC_ERR_INVALID, "a batch needs at least one box");
    FC_REQUIRE(prm.precision == FC_FP64 || prm.precision == FC_FP32_MIXED,
               FC_ERR_INVALID, "unknown precision");
    FC_REQUIRE(prm.lanes >= 0 && prm.lanes <= 32, FC_ERR_INVALID,
               "lanes must be 0 (tuned) to 32");
    size_t free0 = 0, total = 0;
    FC_CUDA(cudaMemGetInfo(&free0, &total));
    for (int i = 0; i < nboxes; ++i) {
      BatchBox b;
      for (int a = 0; a < 3; ++a) {
        FC_REQUIRE(bx[i].shape[a] > 0, FC_ERR_INVALID, "box shape must be positive");
        b.shape[a] = bx[i].shape[a];
      }
      FC_REQUIRE(bx[i].cell_size > 0, FC_ERR_INVALID, "cell_size must be positive");
      FC_REQUIRE(bx[i].n >= 0, FC_ERR_INVALID, "negative particle count");
      FC_REQUIRE(bx[i].n == 0 || bx[i].posw_device, FC_ERR_INVALID,
                 "null particle array");
      b.cell = bx[i].cell_size;
      b.posw = bx[i].posw_device;
      b.n = bx[i].n;
      boxes.push_back(b);
    }
    FC_CUDA(cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking));
    FC_CUDA(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
    FC_CUDA(cudaEventCreate(&t0));
    FC_CUDA(cudaEventCreate(&t1));
    const double zero[3] = {0, 0, 0};
    for (auto &b : boxes) {
      // Grids of the batch's precision: FP32 cells in the FP32-mixed form.
      grids.emplace_back(new Grid(b.shape, zero, b.cell, prm.precision));
      Grid *g = grids.back().get();
      mas.push_back(assignor_new(g, prm.scheme, true));
      assignor_prepare_graph(mas.back(), b.n, g->stream);
      corrs.push_back(correlator_new(FC_PERIODIC, b.shape, b.cell, nullptr,
                                     prm.window, prm.rmax, prm.dr, prm.kmax,
                                     prm.dk, prm.maxell, prm.precision));
      correlator_make_deferred(corrs.back());
      ls_norm.push_back(LaunchShape{256, 64});
    }
    for (auto *c : corrs) correlator_hist_work(c, items, folds);
    d_items.resize(std::max<size_t>(items.size(), 1) * sizeof(HistItem));
    d_folds.resize(std::max<size_t>(folds.size(), 1) * sizeof(FoldItem));
    d_partials.resize(std::max<size_t>(items.size(), 1) * sizeof(double));
    if (!items.empty())
      FC_CUDA(cudaMemcpy(d_items.get(), items.data(),
                         items.size() * sizeof(HistItem), cudaMemcpyHostToDevice));
    if (!folds.empty())
      FC_CUDA(cudaMemcpy(d_folds.get(), folds.data(),
                         folds.size() * sizeof(FoldItem), cudaMemcpyHostToDevice));
    FC_CUDA(cudaDeviceSynchronize());
    tune_kernels();
    choose_lanes_and_capture();
    size_t free1 = 0;
    FC_CUDA(cudaMemGetInfo(&free1, &total));
    device_bytes = free0 > free1 ? free0 - free1 : 0;
  }

  ~Batch() {
    if (main) cudaStreamSynchronize(main);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto *c : corrs) correlator_delete(c);
    for (auto *a : mas) assignor_delete(a);
    grids.clear();
    for (auto s : lanes) cudaStreamDestroy(s);
    for (auto e : join_ev) cudaEventDestroy(e);
    if (fork_ev) cudaEventDestroy(fork_ev);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (main) cudaStreamDestroy(main);
  }

  // ---------------------------------------------------------------- work
  template <typename T>
  void norm_pad(int i, cudaStream_t s) {
    const BatchBox &b = boxes[i];
    const size_t nrows = (size_t)b.shape[0] * b.shape[1];
    const int n2p = 2 * (b.shape[2] / 2 + 1);
    const LaunchShape &ls = ls_norm[i];
    const unsigned blocks =
        (unsigned)std::min<size_t>(nrows, (size_t)sm_count() * ls.waves);
    T *work = static_cast<T *>(correlator_work(corrs[i]));
    const Grid *g = grids[i].get();
    if (g->fp32())
      k_norm_pad<float, T><<<blocks, ls.threads, 0, s>>>(
          static_cast<const float *>(g->raw()), work, b.shape[0], b.shape[1],
          b.shape[2], n2p, assignor_totals(mas[i]), (double)g->size());
    else
      k_norm_pad<double, T><<<blocks, ls.threads, 0, s>>>(
          g->ptr(), work, b.shape[0], b.shape[1], b.shape[2], n2p,
          assignor_totals(mas[i]), (double)g->size());
    FC_LAUNCH_CHECK();
  }

  void enqueue_box(int i, cudaStream_t s) {
    Grid *g = grids[i].get();
    FC_CUDA(cudaMemsetAsync(g->raw(), 0, g->size() * g->cell_bytes(), s));
    assignor_enqueue_graph(mas[i], boxes[i].posw, boxes[i].n, s);
    if (fp64())
      norm_pad<double>(i, s);
    else
      norm_pad<float>(i, s);
    correlator_set_stream(corrs[i], s);
    correlator_enqueue_prepared(corrs[i]);
  }

  void enqueue_hist(cudaStream_t s) {
    if (!items.empty()) {
      k_batch_chunks<<<hist_blocks, kHistThreads, 0, s>>>(
          d_items.as<HistItem>(), (int)items.size(), d_partials.as<double>());
      FC_LAUNCH_CHECK();
    }
    if (!folds.empty()) {
      k_batch_fold<<<grid_for(folds.size(), 128), 128, 0, s>>>(
          d_folds.as<FoldItem>(), (int)folds.size(), d_partials.as<double>());
      FC_LAUNCH_CHECK();
    }
  }

  // ---------------------------------------------------------------- tuning
  // Grid-stride kernels, per distinct box shape: the fastest (threads,
  // waves) of the candidates on the first box of that shape.
  void tune_kernels() {
    std::map<std::string, int> first;  // shape key -> representative box
    for (int i = 0; i < (int)boxes.size(); ++i) {
      std::string k = tune::shape_key("box", fp64(), boxes[i].shape);
      if (!first.count(k)) first[k] = i;
    }
    const char *names[4] = {"norm", "abs2", "ksub", "rsub"};
    for (auto &kv : first) {
      const int rep = kv.second;
      std::pair<int, int> best[4];
      for (int which = 0; which < 4; ++which) {
        const std::string key = tune::shape_key(names[which], fp64(), boxes[rep].shape);
        if (tune::get(key, &best[which])) continue;
        if (!prm.tune) {
          best[which] = which == 0 ? std::make_pair(256, 64) : std::make_pair(256, 8);
          continue;
        }
        float best_ms = 1e30f;
        for (int th : kThreadChoices)
          for (int wv : kWaveChoices) {
            const int waves = which == 0 ? wv * 4 : wv;  // rows kernel
            float ms;
            if (which == 0) {
              ls_norm[rep] = LaunchShape{th, waves};
              ms = time_on(main, [&] {
                if (fp64()) norm_pad<double>(rep, main);
                else norm_pad<float>(rep, main);
              });
            } else {
              CorrShapes cs = correlator_shapes(corrs[rep]);
              LaunchShape *ls = which == 1 ? cs.abs2 : which == 2 ? cs.ksub : cs.rsub;
              *ls = LaunchShape{th, waves};
              ms = time_on(main, [&] {
                correlator_time_kernels(corrs[rep], which - 1, main);
              });
            }
            if (ms < best_ms) {
              best_ms = ms;
              best[which] = {th, waves};
            }
          }
        tune::put(key, best[which]);
      }
      // Apply to every box of this shape.
      for (int i = 0; i < (int)boxes.size(); ++i) {
        if (tune::shape_key("box", fp64(), boxes[i].shape) != kv.first) continue;
        ls_norm[i] = LaunchShape{best[0].first, best[0].second};
        CorrShapes cs = correlator_shapes(corrs[i]);
        *cs.abs2 = LaunchShape{best[1].first, best[1].second};
        *cs.ksub = LaunchShape{best[2].first, best[2].second};
        *cs.rsub = LaunchShape{best[3].first, best[3].second};
      }
    }
    // Histogram CTAs.
    char key[64];
    std::snprintf(key, sizeof(key), "hist %s items%zu", fp64() ? "f64" : "f32",
                  items.size());
    std::pair<int, int> hb;
    if (tune::get(key, &hb)) {
      hist_blocks = hb.first;
    } else if (!prm.tune) {
      hist_blocks = sm_count() * 4;
    } else {
      float best_ms = 1e30f;
      for (int w : {1, 2, 4, 8, 16}) {
        hist_blocks = sm_count() * w;
        const float ms = time_on(main, [&] { enqueue_hist(main); });
        if (ms < best_ms) {
          best_ms = ms;
          hb = {hist_blocks, 0};
        }
      }
      hist_blocks = hb.first;
      tune::put(key, hb);
    }
    FC_CUDA(cudaStreamSynchronize(main));
  }

  void assign_lanes(int n) {
    std::vector<int> order(boxes.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    auto cost = [&](int i) {
      const double cells = (double)boxes[i].shape[0] * boxes[i].shape[1] *
                           boxes[i].shape[2];
      return cells * (fp64() ? 60.0 : 36.0) + (double)boxes[i].n * 100.0;
    };
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<double> load(n, 0.0);
    lane_of.assign(boxes.size(), 0);
    for (int i : order) {
      const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      lane_of[i] = l;
      load[l] += cost(i);
    }
  }

  void capture(int n) {
    while ((int)lanes.size() < n) {
      cudaStream_t s;
      FC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      lanes.push_back(s);
      cudaEvent_t e;
      FC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      join_ev.push_back(e);
    }
    if (exec) {
      FC_CUDA(cudaGraphExecDestroy(exec));
      exec = nullptr;
    }
    if (graph) {
      FC_CUDA(cudaGraphDestroy(graph));
      graph = nullptr;
    }
    assign_lanes(n);
    nlanes = n;
    const unsigned long long before = launch_counter().load();
    FC_CUDA(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
    try {
      FC_CUDA(cudaEventRecord(fork_ev, main));
      for (int l = 0; l < n; ++l) FC_CUDA(cudaStreamWaitEvent(lanes[l], fork_ev, 0));
      for (int l = 0; l < n; ++l)
        for (int i = 0; i < (int)boxes.size(); ++i)
          if (lane_of[i] == l) enqueue_box(i, lanes[l]);
      for (int l = 0; l < n; ++l) {
        FC_CUDA(cudaEventRecord(join_ev[l], lanes[l]));
        FC_CUDA(cudaStreamWaitEvent(main, join_ev[l], 0));
      }
      enqueue_hist(main);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(main, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    FC_CUDA(cudaStreamEndCapture(main, &graph));
    own_kernels = launch_counter().load() - before;
    FC_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    FC_CUDA(cudaGraphUpload(exec, main));
    graph_nodes = 0;
    FC_CUDA(cudaGraphGetNodes(graph, nullptr, &graph_nodes));
    std::vector<cudaGraphNode_t> nodes(graph_nodes);
    FC_CUDA(cudaGraphGetNodes(graph, nodes.data(), &graph_nodes));
    kernel_nodes = 0;
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      FC_CUDA(cudaGraphNodeGetType(nd, &t));
      if (t == cudaGraphNodeTypeKernel) ++kernel_nodes;
    }
  }

  void choose_lanes_and_capture() {
    char key[64];
    std::snprintf(key, sizeof(key), "lanes %s boxes%zu", fp64() ? "f64" : "f32",
                  boxes.size());
    if (prm.lanes > 0) {
      capture(prm.lanes);
      return;
    }
    std::pair<int, int> v;
    if (tune::get(key, &v)) {
      capture(v.first);
      return;
    }
    if (!prm.tune) {
      capture(std::min<int>(4, (int)boxes.size()));
      return;
    }
    int best_n = 1;
    float best_ms = 1e30f;
    for (int n : {1, 2, 4, 8, 16}) {
      if (n > (int)boxes.size()) break;
      capture(n);
      const float ms = time_on(main, [&] { FC_CUDA(cudaGraphLaunch(exec, main)); }, 2);
      if (ms < best_ms) {
        best_ms = ms;
        best_n = n;
      }
    }
    tune::put(key, {best_n, 0});
    if (best_n != nlanes) capture(best_n);
  }

  void launch() {
    FC_CUDA(cudaEventRecord(t0, main));
    FC_CUDA(cudaGraphLaunch(exec, main));
    FC_CUDA(cudaEventRecord(t1, main));
  }

  void wait() {
    FC_CUDA(cudaStreamSynchronize(main));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, t0, t1) == cudaSuccess) last_seconds = ms * 1e-3;
  }
};

}  // namespace fc

using namespace fc;

namespace {
Batch *as_batch(fc_batch *b) {
  FC_REQUIRE(b, FC_ERR_INVALID, "null batch handle");
  return reinterpret_cast<Batch *>(b);
}
Batch *as_batch(const fc_batch *b) {
  FC_REQUIRE(b, FC_ERR_INVALID, "null batch handle");
  return reinterpret_cast<Batch *>(const_cast<fc_batch *>(b));
}
int check_box(const Batch *b, int box) {
  FC_REQUIRE(box >= 0 && box < (int)b->boxes.size(), FC_ERR_RANGE,
             "box index out of range");
  return box;
}
}  // namespace

extern "C" {

int fc_batch_params_default(fc_batch_params *p) {
  return guard([&] {
    FC_REQUIRE(p, FC_ERR_INVALID, "null argument");
    std::memset(p, 0, sizeof(*p));
    p->scheme = FC_CLOUD_IN_CELL;
    p->window = FC_NO_CORRECTION;
    p->rmax = 200.0;
    p->dr = 5.0;
    p->kmax = 0.1;
    p->dk = 0.005;
    p->maxell = 2;
    p->precision = FC_FP32_MIXED;
    p->lanes = 0;
    p->tune = 1;
  });
}

int fc_batch_create(const fc_batch_box *boxes, int nboxes,
                    const fc_batch_params *params, fc_batch **out) {
  return guard([&] {
    FC_REQUIRE(boxes && params && out, FC_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<Batch> b(new Batch(*params));
    b->init(boxes, nboxes);
    *out = reinterpret_cast<fc_batch *>(b.release());
  });
}

int fc_batch_destroy(fc_batch *batch) {
  return guard([&] { delete reinterpret_cast<Batch *>(batch); });
}

int fc_batch_run(fc_batch *batch, double *seconds) {
  return guard([&] {
    Batch *b = as_batch(batch);
    b->launch();
    b->wait();
    if (seconds) *seconds = b->last_seconds;
  });
}

int fc_batch_launch(fc_batch *batch) {
  return guard([&] { as_batch(batch)->launch(); });
}

int fc_batch_wait(fc_batch *batch, double *seconds) {
  return guard([&] {
    Batch *b = as_batch(batch);
    b->wait();
    if (seconds) *seconds = b->last_seconds;
  });
}

int fc_batch_info(const fc_batch *batch, fc_batch_info_t *info) {
  return guard([&] {
    FC_REQUIRE(info, FC_ERR_INVALID, "null argument");
    const Batch *b = as_batch(batch);
    info->nboxes = (int)b->boxes.size();
    info->lanes = b->nlanes;
    info->hist_blocks = b->hist_blocks;
    info->graph_nodes = (int64_t)b->graph_nodes;
    info->kernel_nodes = (int64_t)b->kernel_nodes;
    info->own_kernel_nodes = (int64_t)b->own_kernels;
    info->hist_items = (int64_t)b->items.size();
    info->device_bytes = (int64_t)b->device_bytes;
  });
}

int fc_batch_box_dims(const fc_batch *batch, int box, int *nrows, int *nr,
                      int *nk) {
  return guard([&] {
    Batch *b = as_batch(batch);
    correlator_dims(b->corrs[check_box(b, box)], nrows, nr, nk);
  });
}

int fc_batch_results(const fc_batch *batch, int box, double *rbins,
                     int *rcounts, double *rhist, double *kbins, int *kcounts,
                     double *khist, double *zerolag) {
  return guard([&] {
    Batch *b = as_batch(batch);
    FC_CUDA(cudaStreamSynchronize(b->main));
    correlator_results(b->corrs[check_box(b, box)], rbins, rcounts, rhist,
                       kbins, kcounts, khist, zerolag);
  });
}

int fc_batch_box_stats(const fc_batch *batch, int box, fc_assign_stats *s) {
  return guard([&] {
    FC_REQUIRE(s, FC_ERR_INVALID, "null argument");
    Batch *b = as_batch(batch);
    const int i = check_box(b, box);
    FC_CUDA(cudaStreamSynchronize(b->main));
    double tot[2];
    unsigned long long added = 0;
    FC_CUDA(cudaMemcpy(tot, assignor_totals(b->mas[i]), sizeof(tot),
                       cudaMemcpyDeviceToHost));
    FC_CUDA(cudaMemcpy(&added, assignor_counts(b->mas[i]), sizeof(added),
                       cudaMemcpyDeviceToHost));
    std::memset(s, 0, sizeof(*s));
    s->num_added = added;
    s->num_skipped = (uint64_t)b->boxes[i].n - added;
    s->totw = tot[0];
    s->totwsq = tot[1];
  });
}

int fc_tune_export(const char *path) {
  return guard([&] {
    FC_REQUIRE(path, FC_ERR_INVALID, "null path");
    std::ofstream f(path);
    FC_REQUIRE(f.good(), FC_ERR_INVALID, std::string("cannot write ") + path);
    f << "# fftcorr_b200 launch tuning v1: kernel precision size a b\n";
    std::lock_guard<std::mutex> g(tune::mu);
    for (auto &kv : tune::table())
      f << kv.first << " " << kv.second.first << " " << kv.second.second << "\n";
  });
}

int fc_tune_import(const char *path) {
  return guard([&] {
    FC_REQUIRE(path, FC_ERR_INVALID, "null path");
    std::ifstream f(path);
    FC_REQUIRE(f.good(), FC_ERR_INVALID, std::string("cannot read ") + path);
    std::string line;
    std::vector<std::pair<std::string, std::pair<int, int>>> rows;
    while (std::getline(f, line)) {
      if (line.empty() || line[0] == '#') continue;
      std::istringstream ss(line);
      std::string kernel, prec, size;
      int a = 0, b = 0;
      FC_REQUIRE(static_cast<bool>(ss >> kernel >> prec >> size >> a >> b),
                 FC_ERR_INVALID, "malformed tuning line: " + line);
      FC_REQUIRE(a > 0 && b >= 0, FC_ERR_INVALID, "bad tuning values: " + line);
      rows.push_back({kernel + " " + prec + " " + size, {a, b}});
    }
    for (auto &r : rows) tune::put(r.first, r.second);
  });
}

int fc_tune_forget(void) {
  return guard([&] {
    std::lock_guard<std::mutex> g(tune::mu);
    tune::table().clear();
  });
}

int fc_tune_count(int *n) {
  return guard([&] {
    FC_REQUIRE(n, FC_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> g(tune::mu);
    *n = (int)tune::table().size();
  });
}

}  // extern "C"
