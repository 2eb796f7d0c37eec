// fc_serve.cu -- the serving form: a request loop over correlation jobs with
// continuous batching and admission by HBM footprint.
//
// A job is what a user script or the reference CLI does for one catalog
// (cc/fftcorr.cc:233-463): assign the data (and for a survey the randoms,
// as D - alpha R with alpha = sum w_D / sum w_R, the randoms negated as in
// fftcorr/fftcorr.py:538), normalise a periodic grid by its mean
// (cc/fftcorr.cc:369-375), and autocorrelate (correlator.h:273-357 or
// 406-497); a survey job asked for xi also correlates the RR grid.
//
// The server runs `slots` worker threads.  Each free worker takes the first
// queued job that fits the memory budget (a job may pass one that does not
// fit, up to max_bypass times per waiting job, so small jobs keep flowing
// while a large one waits for memory), so jobs that arrive while others run
// are admitted as soon as a slot and memory free up, and their kernels
// overlap on the device (each job's objects own their own streams).
//
// Grids (with their assignors) and correlators stay resident after a job,
// keyed by configuration, and are reused by later jobs of the same
// configuration: FFT plans, twiddle tables, subgrid bin indices and buffers
// are built once.  Memory accounting is by footprint estimate; idle resident
// objects are evicted least recently used first when a new job needs room.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "fc_internal.h"

namespace fc {
namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Tables {
  std::vector<double> rbins, rhist, kbins, khist;
  std::vector<int> rcounts, kcounts;
  double zerolag = 0.0;
};

// A resident object: a grid with its assignor, or a correlator.
struct Resident {
  std::string key;
  size_t bytes = 0;
  bool in_use = false;
  uint64_t last_used = 0;
  int64_t capacity = 0;  // particles the assignor is sized for
  std::unique_ptr<Grid> grid;
  Assignor *ma = nullptr;
  Correlator *corr = nullptr;
  ~Resident() {
    if (corr) correlator_delete(corr);
    if (ma) assignor_delete(ma);
  }
};

struct Job {
  uint64_t ticket = 0;
  fc_job spec;
  size_t footprint = 0;
  int state = 0;  // 0 queued, 1 running, 2 done
  int status = 0;
  std::string message;
  double t_submit = 0, t_start = 0, t_end = 0;
  int bypassed = 0;
  int nrows = 0, nr = 0, nk = 0;
  Tables nn, rr;
  bool has_rr = false;
  fc_assign_stats data_stats{}, rand_stats{};
  double phase[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // Resources held while running.
  std::vector<Resident *> held;
  size_t transient = 0;
};

std::string grid_key(const fc_job &j) {
  std::ostringstream s;
  s.precision(17);
  s << "grid " << j.shape[0] << "x" << j.shape[1] << "x" << j.shape[2] << " "
    << j.cell << " " << j.posmin[0] << "," << j.posmin[1] << "," << j.posmin[2]
    << " s" << j.scheme << " p" << (j.kind == FC_PERIODIC) << " f"
    << j.precision;
  return s.str();
}

std::string corr_key(const fc_job &j) {
  std::ostringstream s;
  s.precision(17);
  s << "corr k" << j.kind << " " << j.shape[0] << "x" << j.shape[1] << "x"
    << j.shape[2] << " " << j.cell << " " << j.posmin[0] << "," << j.posmin[1]
    << "," << j.posmin[2] << " w" << j.window << " " << j.rmax << " " << j.dr
    << " " << j.kmax << " " << j.dk << " l" << j.maxell << " p" << j.precision;
  return s.str();
}

// A job's grids have the cells of its precision (FP32 for FP32-mixed jobs).
size_t grid_bytes(const fc_job &j) {
  const size_t cell = j.precision == FC_FP32_MIXED ? sizeof(float) : sizeof(double);
  return (size_t)j.shape[0] * j.shape[1] * j.shape[2] * cell +
         (2 * kSumBlocks + 2) * sizeof(double);
}

int64_t max_particles(const fc_job &j) {
  return std::max(j.data.n, j.kind == FC_SURVEY ? j.randoms.n : (int64_t)0);
}

size_t stage_rows_bytes(int64_t n) { return ((size_t)n * 32 + 255) / 256 * 256; }

// Device bytes of a worker's catalog staging for job j: every catalog of
// the job (a survey's data and randoms side by side, so the randoms can be
// copied in while the data are assigned) plus scratch for cluster centres.
size_t job_stage_bytes(const fc_job &j) {
  const size_t cs = std::max(catalog_scratch_bytes(j.data),
                             j.kind == FC_SURVEY ? catalog_scratch_bytes(j.randoms) : 0);
  return stage_rows_bytes(j.data.n) +
         (j.kind == FC_SURVEY ? stage_rows_bytes(j.randoms.n) : 0) + cs;
}

void validate(const fc_job &j) {
  FC_REQUIRE(j.kind == FC_PERIODIC || j.kind == FC_SURVEY, FC_ERR_INVALID,
             "unknown job kind");
  FC_REQUIRE(j.precision == FC_FP64 || j.precision == FC_FP32_MIXED,
             FC_ERR_INVALID, "unknown precision");
  FC_REQUIRE(j.scheme >= 0 && j.scheme <= 3, FC_ERR_INVALID,
             "unknown distribution scheme");
  FC_REQUIRE(j.scheme != 2 || assignor_has_d12(), FC_ERR_UNSUPPORTED,
             "this build has no D12 wavelet table");
  for (int i = 0; i < 3; ++i)
    FC_REQUIRE(j.shape[i] > 0, FC_ERR_INVALID, "grid shape must be positive");
  FC_REQUIRE(j.cell > 0, FC_ERR_INVALID, "cell size must be positive");
  FC_REQUIRE(j.data.n >= 0 && j.data.n < (int64_t)0xffffffffll, FC_ERR_INVALID,
             "data count out of range");
  if (j.kind == FC_SURVEY)
    FC_REQUIRE(j.randoms.n > 0 && j.randoms.n < (int64_t)0xffffffffll,
               FC_ERR_INVALID, "a survey job needs randoms");
}

}  // namespace

// Device bytes a job needs: its grids with assignors, its correlator and
// the staging copy of the largest catalog.
size_t job_footprint(const fc_job &j) {
  const int ngrids = j.kind == FC_SURVEY ? 2 : 1;
  size_t b = ngrids * (grid_bytes(j) + assignor_bytes(j.shape, max_particles(j)));
  b += correlator_footprint(j.kind, j.shape, j.cell, j.rmax, j.kmax, j.maxell,
                            j.precision);
  b += job_stage_bytes(j);
  return b;
}

struct Server {
  size_t budget;
  int slots;
  int max_bypass;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job *> queue;
  std::map<uint64_t, std::unique_ptr<Job>> jobs;
  std::list<std::unique_ptr<Resident>> resident;
  size_t bytes_resident = 0, bytes_transient = 0, peak_bytes = 0;
  uint64_t next_ticket = 1, clock = 0;
  int running = 0, peak_running = 0;
  uint64_t completed = 0, admitted_out_of_order = 0, evictions = 0;
  bool stopping = false;
  std::vector<std::thread> workers;
  // Per-worker catalog staging, kept between jobs (grows only; accounted in
  // bytes_resident).
  std::vector<std::unique_ptr<DeviceBuffer>> stage;
  std::vector<size_t> stage_bytes;
  // Per-worker stream for catalog copies (or generation) and the events
  // that mark each catalog in.
  std::vector<cudaStream_t> copy_stream;
  std::vector<cudaEvent_t> data_in, randoms_in;

  Server(size_t budget_, int slots_, int max_bypass_)
      : budget(budget_), slots(slots_), max_bypass(max_bypass_) {
    FC_REQUIRE(slots >= 1 && slots <= 64, FC_ERR_INVALID, "slots must be 1..64");
    FC_REQUIRE(budget > 0, FC_ERR_INVALID, "budget must be positive");
    FC_CUDA(cudaGetDevice(&device));
    copy_stream.assign(slots, nullptr);
    data_in.assign(slots, nullptr);
    randoms_in.assign(slots, nullptr);
    try {
      for (int i = 0; i < slots; ++i) {
        stage.emplace_back(new DeviceBuffer);
        stage_bytes.push_back(0);
        FC_CUDA(cudaStreamCreateWithFlags(&copy_stream[i], cudaStreamNonBlocking));
        FC_CUDA(cudaEventCreateWithFlags(&data_in[i], cudaEventDisableTiming));
        FC_CUDA(cudaEventCreateWithFlags(&randoms_in[i], cudaEventDisableTiming));
      }
    } catch (...) {
      release_streams();
      throw;
    }
    for (int i = 0; i < slots; ++i) workers.emplace_back([this, i] { worker(i); });
  }

  void release_streams() {
    for (auto &x : copy_stream)
      if (x) cudaStreamDestroy(x), x = nullptr;
    for (auto &e : data_in)
      if (e) cudaEventDestroy(e), e = nullptr;
    for (auto &e : randoms_in)
      if (e) cudaEventDestroy(e), e = nullptr;
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> g(mu);
      stopping = true;
    }
    cv_work.notify_all();
    for (auto &t : workers) t.join();
    for (auto x : copy_stream)
      if (x) cudaStreamSynchronize(x);
    release_streams();
  }

  uint64_t submit(const fc_job &spec) {
    validate(spec);
    const size_t fp = job_footprint(spec);
    if (fp > budget)
      FC_THROW(FC_ERR_ADMISSION,
               "job needs " + std::to_string(fp) + " bytes of device memory, "
               "more than the server's budget of " + std::to_string(budget));
    std::unique_ptr<Job> j(new Job);
    j->spec = spec;
    j->footprint = fp;
    j->t_submit = now_s();
    std::lock_guard<std::mutex> g(mu);
    FC_REQUIRE(!stopping, FC_ERR_STATE, "server is shutting down");
    j->ticket = next_ticket++;
    const uint64_t t = j->ticket;
    queue.push_back(j.get());
    jobs[t] = std::move(j);
    cv_work.notify_one();
    return t;
  }

  // ------------------------------------------------------------ admission
  // Under the lock: the resources job j would take, or false if they do
  // not fit now.  On success they are marked in use (new ones are created
  // by the worker outside the lock) and accounted.
  bool try_admit(Job *j, int slot) {
    const fc_job &s = j->spec;
    const int ngrids = s.kind == FC_SURVEY ? 2 : 1;
    const std::string gk = grid_key(s), ck = corr_key(s);
    const int64_t need_n = max_particles(s);
    std::vector<Resident *> reuse;
    size_t extra = 0;
    int grids_found = 0;
    Resident *corr = nullptr;
    for (auto &r : resident) {
      if (r->in_use) continue;
      if (grids_found < ngrids && r->key == gk) {
        reuse.push_back(r.get());
        ++grids_found;
        if (r->capacity < need_n)
          extra += assignor_bytes(s.shape, need_n) - assignor_bytes(s.shape, r->capacity);
      } else if (!corr && r->key == ck) {
        corr = r.get();
        reuse.push_back(r.get());
      }
    }
    const size_t gb = grid_bytes(s) + assignor_bytes(s.shape, need_n);
    extra += (size_t)(ngrids - grids_found) * gb;
    if (!corr)
      extra += correlator_footprint(s.kind, s.shape, s.cell, s.rmax, s.kmax,
                                    s.maxell, s.precision);
    // The worker's staging grows to the largest catalog it has seen.
    const size_t need_stage = job_stage_bytes(s);
    const size_t grow_stage = need_stage > stage_bytes[slot] ? need_stage - stage_bytes[slot] : 0;
    extra += grow_stage;
    // Idle residents not reused here can be evicted.
    size_t evictable = 0;
    for (auto &r : resident)
      if (!r->in_use && std::find(reuse.begin(), reuse.end(), r.get()) == reuse.end())
        evictable += r->bytes;
    const size_t used = bytes_resident + bytes_transient;
    if (used - evictable + extra > budget) return false;
    // Evict least recently used idle objects until the job fits.
    while (used_bytes() + extra > budget) {
      Resident *victim = nullptr;
      for (auto &r : resident)
        if (!r->in_use && std::find(reuse.begin(), reuse.end(), r.get()) == reuse.end() &&
            (!victim || r->last_used < victim->last_used))
          victim = r.get();
      if (!victim) break;
      bytes_resident -= victim->bytes;
      ++evictions;
      resident.remove_if([&](const std::unique_ptr<Resident> &p) { return p.get() == victim; });
    }
    // Mark and account.
    for (Resident *r : reuse) {
      r->in_use = true;
      r->last_used = ++clock;
      if (r->grid && r->capacity < need_n) {
        const size_t grow = assignor_bytes(s.shape, need_n) - assignor_bytes(s.shape, r->capacity);
        r->bytes += grow;
        bytes_resident += grow;
        r->capacity = need_n;
      }
    }
    j->held = reuse;
    for (int i = grids_found; i < ngrids; ++i) {
      std::unique_ptr<Resident> r(new Resident);
      r->key = gk;
      r->bytes = gb;
      r->capacity = need_n;
      r->in_use = true;
      r->last_used = ++clock;
      bytes_resident += gb;
      j->held.push_back(r.get());
      resident.push_back(std::move(r));
    }
    if (!corr) {
      std::unique_ptr<Resident> r(new Resident);
      r->key = ck;
      r->bytes = correlator_footprint(s.kind, s.shape, s.cell, s.rmax, s.kmax,
                                      s.maxell, s.precision);
      r->in_use = true;
      r->last_used = ++clock;
      bytes_resident += r->bytes;
      j->held.push_back(r.get());
      resident.push_back(std::move(r));
    }
    if (grow_stage) {
      stage_bytes[slot] += grow_stage;
      bytes_resident += grow_stage;
    }
    j->transient = 0;
    peak_bytes = std::max(peak_bytes, used_bytes());
    return true;
  }

  size_t used_bytes() const { return bytes_resident + bytes_transient; }

  Job *next_job(int slot) {
    for (size_t i = 0; i < queue.size(); ++i) {
      Job *j = queue[i];
      if (try_admit(j, slot)) {
        queue.erase(queue.begin() + i);
        if (i > 0) ++admitted_out_of_order;
        for (size_t k = 0; k < i; ++k) ++queue[k]->bypassed;
        return j;
      }
      // Jobs behind one that has been passed too often must wait for it.
      if (j->bypassed >= max_bypass) break;
    }
    return nullptr;
  }

  // ---------------------------------------------------------------- work
  void worker(int slot) {
    cudaSetDevice(device);
    for (;;) {
      Job *j = nullptr;
      {
        std::unique_lock<std::mutex> g(mu);
        // Admissible jobs are drained before a stop takes effect.
        cv_work.wait(g, [&] {
          j = next_job(slot);
          return j != nullptr || (stopping && queue.empty());
        });
        if (!j) return;
        j->state = 1;
        j->t_start = now_s();
        ++running;
        peak_running = std::max(peak_running, running);
      }
      try {
        run(j, slot);
      } catch (const Error &e) {
        j->status = e.code;
        j->message = e.what();
      } catch (const std::bad_alloc &) {
        j->status = FC_ERR_ALLOC;
        j->message = "host allocation failed";
      } catch (const std::exception &e) {
        j->status = FC_ERR_CUDA;
        j->message = e.what();
      }
      {
        std::lock_guard<std::mutex> g(mu);
        for (Resident *r : j->held) {
          r->in_use = false;
          r->last_used = ++clock;
        }
        // A failed job may have left an object half built: drop those.
        if (j->status != 0) {
          for (Resident *r : j->held) {
            bytes_resident -= r->bytes;
            resident.remove_if([&](const std::unique_ptr<Resident> &p) { return p.get() == r; });
          }
        }
        j->held.clear();
        bytes_transient -= j->transient;
        j->transient = 0;
        j->t_end = now_s();
        j->state = 2;
        --running;
        ++completed;
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }

  static void read_tables(Correlator *c, Job *j, Tables &t) {
    correlator_dims(c, &j->nrows, &j->nr, &j->nk);
    t.rbins.resize(j->nr);
    t.kbins.resize(j->nk);
    t.rcounts.resize((size_t)j->nrows * j->nr);
    t.kcounts.resize((size_t)j->nrows * j->nk);
    t.rhist.resize((size_t)j->nrows * j->nr);
    t.khist.resize((size_t)j->nrows * j->nk);
    correlator_results(c, t.rbins.data(), t.rcounts.data(), t.rhist.data(),
                       t.kbins.data(), t.kcounts.data(), t.khist.data(),
                       &t.zerolag);
  }

  void run(Job *j, int slot) {
    const fc_job &s = j->spec;
    double t = now_s();
    auto lap = [&](int k) {
      const double t1 = now_s();
      j->phase[k] += t1 - t;
      t = t1;
    };
    const std::string gk = grid_key(s);
    std::vector<Resident *> grids;
    Resident *cr = nullptr;
    for (Resident *r : j->held) {
      if (r->key == gk)
        grids.push_back(r);
      else
        cr = r;
    }
    // Build what is not resident yet.
    for (Resident *r : grids) {
      if (!r->grid) {
        r->grid.reset(new Grid(s.shape, s.posmin, s.cell, s.precision));
        r->ma = assignor_new(r->grid.get(), s.scheme, s.kind == FC_PERIODIC);
      }
    }
    if (!cr->corr)
      cr->corr = correlator_new(s.kind, s.shape, s.cell,
                                s.kind == FC_SURVEY ? s.posmin : nullptr,
                                s.window, s.rmax, s.dr, s.kmax, s.dk, s.maxell,
                                s.precision);
    Grid *ga = grids[0]->grid.get();
    const bool survey = s.kind == FC_SURVEY;
    const size_t cs = std::max(catalog_scratch_bytes(s.data),
                               survey ? catalog_scratch_bytes(s.randoms) : 0);
    const size_t nbuf_d = stage_rows_bytes(s.data.n);
    const size_t nbuf_r = survey ? stage_rows_bytes(s.randoms.n) : 0;
    stage[slot]->resize(std::max<size_t>(nbuf_d + nbuf_r + cs, 32));
    char *st0 = stage[slot]->as<char>();
    double *buf_d = reinterpret_cast<double *>(st0);
    double *buf_r = reinterpret_cast<double *>(st0 + nbuf_d);
    double *scr = reinterpret_cast<double *>(st0 + nbuf_d + nbuf_r);
    cudaStream_t cp = copy_stream[slot];
    // Whatever this job queued is complete when it returns or fails, so the
    // next job on this worker may reuse the staging and the grids.
    struct Drain {
      cudaStream_t s[3];
      ~Drain() {
        for (cudaStream_t x : s)
          if (x) cudaStreamSynchronize(x);
      }
    } drain{{cp, ga->stream, survey ? grids[1]->grid->stream : nullptr}};
    lap(7);
    // Both catalogs come in one after the other on the worker's copy
    // stream, so the randoms' copy (or generation) runs while the data are
    // assigned.  (This worker's previous job is complete: its staging is
    // free.)
    catalog_generate(s.data, buf_d, cp, scr, cs);
    FC_CUDA(cudaEventRecord(data_in[slot], cp));
    if (survey) {
      catalog_generate(s.randoms, buf_r, cp, scr, cs);
      FC_CUDA(cudaEventRecord(randoms_in[slot], cp));
    }
    // Data grid.
    ga->clear();
    assignor_clear(grids[0]->ma);
    FC_CUDA(cudaStreamWaitEvent(ga->stream, data_in[slot], 0));
    FC_CUDA(cudaEventSynchronize(data_in[slot]));
    lap(0);
    assignor_add_device(grids[0]->ma, buf_d, s.data.n);
    assignor_stats(grids[0]->ma, &j->data_stats);
    lap(1);
    fc_grid *ha = reinterpret_cast<fc_grid *>(ga);
    if (s.kind == FC_PERIODIC) {
      // cc/fftcorr.cc:369-375.
      const double mean = j->data_stats.totw / (double)ga->size();
      check(fc_grid_add_scalar(ha, -mean));
      check(fc_grid_multiply_by(ha, 1.0 / mean));
      lap(4);
      correlator_autocorrelate(cr->corr, ga);
      read_tables(cr->corr, j, j->nn);
      lap(5);
      return;
    }
    // Survey: randoms into the second grid, scaled by -alpha.
    Grid *gb = grids[1]->grid.get();
    gb->clear();
    assignor_clear(grids[1]->ma);
    FC_CUDA(cudaStreamWaitEvent(gb->stream, randoms_in[slot], 0));
    FC_CUDA(cudaEventSynchronize(randoms_in[slot]));
    lap(2);
    assignor_add_device(grids[1]->ma, buf_r, s.randoms.n);
    assignor_stats(grids[1]->ma, &j->rand_stats);
    lap(3);
    fc_grid *hb = reinterpret_cast<fc_grid *>(gb);
    FC_REQUIRE(j->rand_stats.totw != 0.0, FC_ERR_INVALID,
               "randoms have zero total weight");
    const double alpha = j->data_stats.totw / j->rand_stats.totw;
    check(fc_grid_multiply_by(hb, -alpha));
    check(fc_grid_axpy(ha, 1.0, hb));
    lap(4);
    correlator_autocorrelate(cr->corr, ga);
    read_tables(cr->corr, j, j->nn);
    lap(5);
    if (s.want_rr) {
      correlator_autocorrelate(cr->corr, gb);
      read_tables(cr->corr, j, j->rr);
      j->has_rr = true;
    }
    lap(6);
  }

  static void check(int rc) {
    if (rc != 0) FC_THROW(rc, last_error_cstr());
  }

  Job *find(uint64_t t) {
    auto it = jobs.find(t);
    FC_REQUIRE(it != jobs.end(), FC_ERR_RANGE, "unknown ticket");
    return it->second.get();
  }
};

}  // namespace fc

using namespace fc;

namespace {
Server *as_server(fc_server *s) {
  FC_REQUIRE(s, FC_ERR_INVALID, "null server handle");
  return reinterpret_cast<Server *>(s);
}
}  // namespace

extern "C" {

int fc_job_init(fc_job *j) {
  return guard([&] {
    FC_REQUIRE(j, FC_ERR_INVALID, "null argument");
    std::memset(j, 0, sizeof(*j));
    j->kind = FC_PERIODIC;
    j->scheme = FC_CLOUD_IN_CELL;
    j->window = FC_NO_CORRECTION;
    j->rmax = 200.0;
    j->dr = 5.0;
    j->kmax = 0.1;
    j->dk = 0.005;
    j->maxell = 2;
    j->precision = FC_FP32_MIXED;
    j->want_rr = 1;
  });
}

int fc_job_footprint(const fc_job *j, size_t *bytes) {
  return guard([&] {
    FC_REQUIRE(j && bytes, FC_ERR_INVALID, "null argument");
    validate(*j);
    *bytes = job_footprint(*j);
  });
}

int fc_server_create(size_t hbm_budget, int slots, int max_bypass,
                     fc_server **out) {
  return guard([&] {
    FC_REQUIRE(out, FC_ERR_INVALID, "null argument");
    *out = reinterpret_cast<fc_server *>(new Server(hbm_budget, slots, max_bypass));
  });
}

int fc_server_destroy(fc_server *server) {
  return guard([&] { delete reinterpret_cast<Server *>(server); });
}

int fc_server_submit(fc_server *server, const fc_job *job, uint64_t *ticket) {
  return guard([&] {
    FC_REQUIRE(job && ticket, FC_ERR_INVALID, "null argument");
    *ticket = as_server(server)->submit(*job);
  });
}

int fc_server_wait(fc_server *server, uint64_t ticket, double timeout_s,
                   int *done) {
  return guard([&] {
    Server *s = as_server(server);
    std::unique_lock<std::mutex> g(s->mu);
    Job *j = s->find(ticket);
    auto pred = [&] { return j->state == 2; };
    if (timeout_s < 0)
      s->cv_done.wait(g, pred);
    else
      s->cv_done.wait_for(g, std::chrono::duration<double>(timeout_s), pred);
    if (done) *done = j->state == 2;
    FC_REQUIRE(j->state == 2, FC_ERR_TIMEOUT, "the job had not finished");
  });
}

int fc_server_job_info(fc_server *server, uint64_t ticket, fc_job_info *info) {
  return guard([&] {
    FC_REQUIRE(info, FC_ERR_INVALID, "null argument");
    Server *s = as_server(server);
    std::lock_guard<std::mutex> g(s->mu);
    Job *j = s->find(ticket);
    std::memset(info, 0, sizeof(*info));
    info->state = j->state;
    info->status = j->status;
    info->queued_s = (j->state >= 1 ? j->t_start : now_s()) - j->t_submit;
    info->run_s = j->state == 2 ? j->t_end - j->t_start : 0.0;
    info->latency_s = j->state == 2 ? j->t_end - j->t_submit : 0.0;
    info->footprint = j->footprint;
    info->nrows = j->nrows;
    info->nr = j->nr;
    info->nk = j->nk;
    info->has_rr = j->has_rr ? 1 : 0;
    for (int k = 0; k < 8; ++k) info->phase_s[k] = j->phase[k];
    info->data = j->data_stats;
    info->randoms = j->rand_stats;
    std::strncpy(info->message, j->message.c_str(), sizeof(info->message) - 1);
  });
}

int fc_server_job_results(fc_server *server, uint64_t ticket, int which,
                          double *rbins, int *rcounts, double *rhist,
                          double *kbins, int *kcounts, double *khist,
                          double *zerolag) {
  return guard([&] {
    Server *s = as_server(server);
    std::lock_guard<std::mutex> g(s->mu);
    Job *j = s->find(ticket);
    FC_REQUIRE(j->state == 2, FC_ERR_STATE, "job has not finished");
    if (j->status != 0) FC_THROW(j->status, j->message);
    FC_REQUIRE(which == 0 || (which == 1 && j->has_rr), FC_ERR_INVALID,
               "no such result (0: NN, 1: RR when asked for)");
    const Tables &t = which == 0 ? j->nn : j->rr;
    auto put = [](auto *dst, const auto &v) {
      if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    put(rbins, t.rbins);
    put(rcounts, t.rcounts);
    put(rhist, t.rhist);
    put(kbins, t.kbins);
    put(kcounts, t.kcounts);
    put(khist, t.khist);
    if (zerolag) *zerolag = t.zerolag;
  });
}

int fc_server_release(fc_server *server, uint64_t ticket) {
  return guard([&] {
    Server *s = as_server(server);
    std::lock_guard<std::mutex> g(s->mu);
    Job *j = s->find(ticket);
    FC_REQUIRE(j->state == 2, FC_ERR_STATE, "job has not finished");
    s->jobs.erase(ticket);
  });
}

int fc_server_stats(fc_server *server, fc_server_stats_t *st) {
  return guard([&] {
    FC_REQUIRE(st, FC_ERR_INVALID, "null argument");
    Server *s = as_server(server);
    std::lock_guard<std::mutex> g(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->queued = (int)s->queue.size();
    st->running = s->running;
    st->peak_running = s->peak_running;
    st->completed = s->completed;
    st->resident_objects = (int)s->resident.size();
    st->bytes_resident = s->bytes_resident;
    st->bytes_transient = s->bytes_transient;
    st->peak_bytes = s->peak_bytes;
    st->budget = s->budget;
    st->admitted_out_of_order = s->admitted_out_of_order;
    st->evictions = s->evictions;
  });
}

}  // extern "C"
