// Autotuner: measured launch choices per size bucket, cached as JSON. No counterpart in the
// reference (its CPU path has nothing to tune). Included by pm3gpu.cu inside its private
// namespace, after run_batch.
//
// Two choices are measured, each between variants that give the same results:
//   batch  CTAs per SM of the persistent SCF launch. One CTA per SM gives each molecule the
//          largest shared-memory eigen workspace (the packed matrix of up to ~230 basis functions
//          stays on chip); two CTAs per SM halve it but double the molecules in flight. The
//          bucket is the batch's largest basis size (the layout is sized for it).
//   large  the whole-GPU Householder reduction as one cooperative launch per panel or as five
//          launches per column replayed from a CUDA graph; bucket = basis size.
// A bucket covers sizes up to its bound; lookups take the smallest tuned bucket that covers the
// size and fall back to the built-in choice (the 90% rule of make_layout, cooperative panels).

constexpr int kTuneBatchBuckets[] = {64, 128, 256};  // coarse: a sample and its full batch share a bucket
constexpr int kTuneLargeBuckets[] = {512, 1024, 2048, 4096, 8192, 16384, 32768, 65536, 131072};

template <size_t N>
int tune_bucket(const int (&b)[N], int v) {
  for (size_t k = 0; k < N; ++k)
    if (v <= b[k]) return b[k];
  return b[N - 1];
}

void tune_store(std::vector<pm3gpu_ctx::Tune>& t, const pm3gpu_ctx::Tune& e) {
  for (pm3gpu_ctx::Tune& x : t)
    if (x.le == e.le) {
      x = e;
      return;
    }
  t.push_back(e);
  std::sort(t.begin(), t.end(), [](const pm3gpu_ctx::Tune& a, const pm3gpu_ctx::Tune& b) { return a.le < b.le; });
}

// Basis size of one molecule (s-only H and He: 1 function, the rest 4).
int tune_nao(const pm3gpu_ctx* c, const int32_t* z, int natom) {
  int n = 0;
  for (int a = 0; a < natom; ++a) n += (z[a] > 0 && z[a] < kMaxZ) ? c->h_elem[z[a]].norb : 0;
  return n;
}

// The batch choice for the molecules of the sample that take the per-CTA path: each candidate
// solves the whole sub-batch twice, the second run's device time counts.
int tune_batch_part(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, const double* xyz,
                    const pm3gpu_options* o) {
  std::vector<int32_t> so(1, 0), sz;
  std::vector<double> sx;
  int nmax = 0;
  for (int m = 0; m < n_mol; ++m) {
    const int na = offs[m + 1] - offs[m];
    const int nao = tune_nao(c, z + offs[m], na);
    if (nao >= c->large_min || nao <= 0) continue;
    nmax = std::max(nmax, nao);
    sz.insert(sz.end(), z + offs[m], z + offs[m + 1]);
    sx.insert(sx.end(), xyz + 3 * (size_t)offs[m], xyz + 3 * (size_t)offs[m + 1]);
    so.push_back((int32_t)sz.size());
  }
  const int nm = (int)so.size() - 1;
  if (nm == 0) return PM3GPU_OK;
  std::vector<pm3gpu_result> res(nm);
  std::vector<double> q(sz.size());
  // Goal "batch time": the whole sample's time, tail included (one batch at a time). Goal
  // "throughput": the time until 90% of the first passes have ended, a measure of the rate in the
  // bulk of a batch, where the tail of one batch overlaps the next when batches are in flight.
  double ms[2] = {0.0, 0.0};
  c->record_jobs = c->tune_goal == PM3GPU_TUNE_THROUGHPUT;
  for (int k = 0; k < 2; ++k) {
    c->force_ctas = k + 1;
    for (int rep = 0; rep < 2; ++rep) {
      const int rc = run_batch(c, nm, so.data(), sz.data(), sx.data(), nullptr, nullptr, o, 0, Want{}, res.data(),
                               q.data(), nullptr, nullptr, nullptr);
      if (rc != PM3GPU_OK) {
        c->force_ctas = 0;
        c->record_jobs = false;
        return rc;
      }
    }
    ms[k] = c->timings[4];
    if (c->record_jobs && c->job_ns.size() > 1) {
      std::vector<unsigned long long> t(c->job_ns.begin(), c->job_ns.end() - 1);
      const unsigned long long t0 = c->job_ns.back();
      std::sort(t.begin(), t.end());
      const size_t k90 = std::min(t.size() - 1, (size_t)(0.9 * (double)t.size()));
      ms[k] = t[k90] > t0 ? 1e-6 * (double)(t[k90] - t0) : ms[k];
    }
  }
  c->force_ctas = 0;
  c->record_jobs = false;
  tune_store(c->tune_batch, {tune_bucket(kTuneBatchBuckets, nmax), ms[1] <= ms[0] ? 2 : 1, ms[0], ms[1]});
  return PM3GPU_OK;
}

// The reduction choice for each size bucket met by the sample's large molecules (first molecule
// per bucket): one Householder reduction of its H_core per candidate.
int tune_large_part(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, const double* xyz) {
  std::vector<int> done;
  for (int m = 0; m < n_mol; ++m) {
    const int na = offs[m + 1] - offs[m];
    const int nao = tune_nao(c, z + offs[m], na);
    if (nao < c->large_min || nao < 3) continue;
    const int b = tune_bucket(kTuneLargeBuckets, nao);
    if (std::find(done.begin(), done.end(), b) != done.end()) continue;
    done.push_back(b);
    CUDA_TRY(c, dgemm_ready(c->device));
    if (!c->lbuf) c->lbuf = new LargeBufs();
    CUDA_TRY(c, c->z.ensure(4 * (size_t)na));
    CUDA_TRY(c, c->xyz.ensure(24 * (size_t)na));
    CUDA_TRY(c, cudaMemcpyAsync(c->z.p, z + offs[m], 4 * (size_t)na, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->xyz.p, xyz + 3 * (size_t)offs[m], 24 * (size_t)na, cudaMemcpyHostToDevice, c->stream));
    LargeSolver S(c, *c->lbuf);
    double ecc = 0.0, t_coop = 0.0, t_multi = 0.0;
    int rc = S.setup(z + offs[m], c->z.as<int32_t>(), c->xyz.as<double>(), na, nao, &ecc);
    if (rc == PM3GPU_OK) rc = S.time_reduction(1, &t_coop);
    if (rc == PM3GPU_OK) rc = S.time_reduction(0, &t_multi);
    c->force_coop = -1;
    if (rc != PM3GPU_OK) return rc;
    tune_store(c->tune_large, {b, t_coop <= t_multi ? 1 : 0, t_coop, t_multi});
  }
  return PM3GPU_OK;
}

int write_tuning(pm3gpu_ctx* c, const char* path) {
  FILE* f = std::fopen(path, "w");
  if (!f) return fail(c, PM3GPU_INVALID_INPUT, std::string("cannot write tuning file ") + path);
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, c->device);
  std::fprintf(f, "{\n  \"device\": \"%s\",\n  \"sms\": %d,\n  \"goal\": \"%s\",\n  \"batch\": [", prop.name, c->sms,
               c->tune_goal == PM3GPU_TUNE_THROUGHPUT ? "throughput" : "batch time");
  for (size_t k = 0; k < c->tune_batch.size(); ++k) {
    const pm3gpu_ctx::Tune& e = c->tune_batch[k];
    std::fprintf(f, "%s\n    {\"nmax_le\": %d, \"ctas_per_sm\": %d, \"ms_1cta\": %.6f, \"ms_2cta\": %.6f}", k ? "," : "",
                 e.le, e.choice, e.ms_a, e.ms_b);
  }
  std::fprintf(f, "\n  ],\n  \"large\": [");
  for (size_t k = 0; k < c->tune_large.size(); ++k) {
    const pm3gpu_ctx::Tune& e = c->tune_large[k];
    std::fprintf(f, "%s\n    {\"n_le\": %d, \"coop\": %d, \"ms_coop\": %.6f, \"ms_multi\": %.6f}", k ? "," : "", e.le,
                 e.choice, e.ms_a, e.ms_b);
  }
  std::fprintf(f, "\n  ]\n}\n");
  const bool ok = std::fclose(f) == 0;
  return ok ? PM3GPU_OK : fail(c, PM3GPU_INVALID_INPUT, std::string("cannot write tuning file ") + path);
}

// Reads the format write_tuning produces: every innermost {...} object with "nmax_le" is a batch
// entry, with "n_le" a large entry; other keys are ignored. With c == nullptr the file is only
// checked (no device is touched).
int read_tuning(pm3gpu_ctx* c, const char* path) {
  FILE* f = std::fopen(path, "r");
  if (!f) return fail(c, PM3GPU_INVALID_INPUT, std::string("cannot read tuning file ") + path);
  std::string text;
  char buf[4096];
  for (size_t got; (got = std::fread(buf, 1, sizeof(buf), f)) > 0;) text.append(buf, got);
  std::fclose(f);
  std::vector<pm3gpu_ctx::Tune> tb, tl;
  for (size_t pos = text.find('{'); pos != std::string::npos; pos = text.find('{', pos + 1)) {
    const size_t end = text.find('}', pos);
    if (end == std::string::npos) break;
    const std::string obj = text.substr(pos, end - pos);
    if (obj.find('{', 1) != std::string::npos) continue;  // not innermost
    auto num = [&](const char* key, double* v) {
      const size_t k = obj.find(std::string("\"") + key + "\"");
      if (k == std::string::npos) return false;
      const size_t colon = obj.find(':', k);
      if (colon == std::string::npos) return false;
      char* stop = nullptr;
      *v = std::strtod(obj.c_str() + colon + 1, &stop);
      return stop != obj.c_str() + colon + 1;
    };
    double le, ch, a = 0.0, b = 0.0;
    // bucket bounds are basis sizes: finite, at least 1 and at most the whole-GPU path's reach
    auto bad_le = [&](double v) { return !std::isfinite(v) || v < 1.0 || v > 1.0e6 || v != std::floor(v); };
    if (num("nmax_le", &le) && num("ctas_per_sm", &ch)) {
      if (bad_le(le)) return fail(c, PM3GPU_INVALID_INPUT, "tuning file: nmax_le must be an integer in 1..1000000");
      num("ms_1cta", &a);
      num("ms_2cta", &b);
      if (ch != 1.0 && ch != 2.0) return fail(c, PM3GPU_INVALID_INPUT, "tuning file: ctas_per_sm must be 1 or 2");
      tb.push_back({(int)le, (int)ch, a, b});
    } else if (num("n_le", &le) && num("coop", &ch)) {
      if (bad_le(le)) return fail(c, PM3GPU_INVALID_INPUT, "tuning file: n_le must be an integer in 1..1000000");
      num("ms_coop", &a);
      num("ms_multi", &b);
      if (ch != 0.0 && ch != 1.0) return fail(c, PM3GPU_INVALID_INPUT, "tuning file: coop must be 0 or 1");
      tl.push_back({(int)le, (int)ch, a, b});
    }
  }
  if (tb.empty() && tl.empty()) return fail(c, PM3GPU_INVALID_INPUT, std::string("no tuning entries in ") + path);
  if (!c) return PM3GPU_OK;
  for (const pm3gpu_ctx::Tune& e : tb) tune_store(c->tune_batch, e);
  for (const pm3gpu_ctx::Tune& e : tl) tune_store(c->tune_large, e);
  return PM3GPU_OK;
}
