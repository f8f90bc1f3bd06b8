// Host side of the post-SCF corrections (pm3-rs src/corrections/mod.rs:129-213): buffers and
// launches of the D3 kernels (d3.cuh) and the H4 / H-H / X kernel (h4.cuh), and their place in the
// single point (src/scf.rs:740-743: the correction joins total_ev and the heat of formation) and the
// gradient (src/gradient.rs:240-262, 324-357: its gradient joins the SCF gradient). Included by
// pm3gpu.cu inside its private namespace, before run_batch.
#pragma once

// A launched correction: which molecules take which terms, and where the results land in the
// context's pinned staging buffer once the stream has reached them.
struct CorrPlan {
  int n_mol = 0, total = 0, nh = 0, nm = 0;
  bool grad = false, any = false;
  std::vector<int32_t> set;
  std::vector<char> is_h, is_m;
  size_t h_e = 0, h_eh = 0, h_em = 0, h_gd3 = 0, h_gh = 0, h_gm = 0;  // offsets into c->h_corr
};

// Enqueue the corrections of the batch in dz / dxyz (device) on the context's stream: molecule m
// takes D3 with the parameter set h_set[m] (0 none, 1 D3Params::pm3_d3, 2 D3Params::pm3_d3h4), when
// h_var[m] is 2 or 3 (PM3-D3H4, PM3-D3H4X) the H4 and H-H terms, 3 adding X, and when h_mmok[m]
// (optional) the MMOK amide term; the results are copied to pinned host memory behind the kernels.
// Nothing waits: corrections_collect reads them after the stream has been synchronised. The terms
// depend on the geometry alone, so a batch launches them ahead of its SCF and they never wait
// behind another stream's persistent SCF kernel at the end of the batch.
int corrections_launch(pm3gpu_ctx* c, int n_mol, const int32_t* h_offs, const int32_t* h_set, const int32_t* h_var,
                       const int32_t* h_mmok, const int32_t* dz, const double* dxyz, bool want_grad, CorrPlan& P) {
  P = CorrPlan{};
  const int total = h_offs[n_mol];
  P.n_mol = n_mol;
  P.total = total;
  P.grad = want_grad;
  if (n_mol <= 0 || total <= 0) return PM3GPU_OK;
  P.set.assign(h_set, h_set + n_mol);
  P.is_h.assign(n_mol, 0);
  P.is_m.assign(n_mol, 0);
  std::vector<int32_t> hmols, mmols;
  bool any_d3 = false;
  for (int m = 0; m < n_mol; ++m) {
    if (h_offs[m + 1] == h_offs[m]) {
      P.set[m] = 0;
      continue;
    }
    any_d3 |= P.set[m] != 0;
    if (h_var[m] >= 2) {
      hmols.push_back(m);
      P.is_h[m] = 1;
    }
    if (h_mmok && h_mmok[m]) {
      mmols.push_back(m);
      P.is_m[m] = 1;
    }
  }
  const int nh = (int)hmols.size(), nm = (int)mmols.size();
  P.nh = nh;
  P.nm = nm;
  P.any = any_d3 || nh || nm;
  if (!P.any) return PM3GPU_OK;
  CUDA_TRY(c, d3_ready(c->device));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));  // no copy of an earlier call still uses the staging
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t A = (size_t)total, M = (size_t)n_mol;
  // host staging (pinned): inputs first, then the outputs the host reads back
  size_t ho = 0;
  auto htake = [&](size_t b) {
    const size_t at = ho;
    ho += up(b);
    return at;
  };
  const size_t h_offs_at = htake(4 * (M + 1)), h_set_at = htake(4 * M), h_var_at = htake(4 * M);
  const size_t h_hm_at = htake(4 * (size_t)nh + 4), h_mm_at = htake(4 * (size_t)nm + 4);
  P.h_e = htake(8 * M);
  P.h_eh = htake(nh ? 24 * M : 0);
  P.h_em = htake(nm ? 8 * M : 0);
  P.h_gd3 = htake(want_grad ? 24 * A : 0);
  P.h_gh = htake(want_grad && nh ? 24 * A : 0);
  P.h_gm = htake(want_grad && nm ? 24 * A : 0);
  if (ho > c->h_corr_bytes) {
    if (c->h_corr) cudaFreeHost(c->h_corr);
    c->h_corr = nullptr;
    c->h_corr_bytes = 0;
    CUDA_TRY(c, cudaHostAlloc(&c->h_corr, ho, cudaHostAllocDefault));
    c->h_corr_bytes = ho;
  }
  char* hb = static_cast<char*>(c->h_corr);
  std::memcpy(hb + h_offs_at, h_offs, 4 * (M + 1));
  std::memcpy(hb + h_set_at, P.set.data(), 4 * M);
  std::memcpy(hb + h_var_at, h_var, 4 * M);
  if (nh) std::memcpy(hb + h_hm_at, hmols.data(), 4 * (size_t)nh);
  if (nm) std::memcpy(hb + h_mm_at, mmols.data(), 4 * (size_t)nm);
  // device buffers
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o += up(b);
    return at;
  };
  const size_t in_bytes = h_mm_at + up(4 * (size_t)nm + 4);  // the input block, copied in one piece
  const size_t o_in = take(in_bytes);
  const size_t o_cn = take(8 * A), o_de = take(8 * A), o_e6 = take(8 * A), o_e8 = take(8 * A);
  const size_t o_gd = take(24 * A), o_g = take(24 * A), o_en = take(8 * M), o_eh = take(24 * M);
  const size_t o_gh = take(nh ? 24 * A : 0), o_ho = take(nh ? 24 * A : 0);
  const size_t o_me = take(nm ? 8 * M : 0), o_mg = take(nm ? 24 * A : 0);
  size_t o_s[16];
  for (int k = 0; k < 16; ++k) o_s[k] = take(nh ? 8 * A : 0);
  CUDA_TRY(c, c->d3buf.ensure(o));
  char* base = c->d3buf.as<char>();
  auto I = [&](size_t off) { return reinterpret_cast<int32_t*>(base + off); };
  auto D = [&](size_t off) { return reinterpret_cast<double*>(base + off); };
  const size_t o_offs = o_in + h_offs_at, o_set = o_in + h_set_at, o_var = o_in + h_var_at;
  const size_t o_hm = o_in + h_hm_at, o_mm = o_in + h_mm_at;
  cudaStream_t s = c->stream;
  CUDA_TRY(c, cudaMemcpyAsync(base + o_in, hb, in_bytes, cudaMemcpyHostToDevice, s));
  const int tb = 128, nb = (total + tb - 1) / tb;
  const int wg = want_grad ? 1 : 0;
  if (any_d3) {
    d3k::cn_kernel<<<nb, tb, 0, s>>>(total, n_mol, I(o_offs), I(o_set), dz, dxyz, D(o_cn));
    d3k::pair_kernel<<<nb, tb, 0, s>>>(total, n_mol, I(o_offs), I(o_set), dz, dxyz, D(o_cn), D(o_e6), D(o_e8),
                                       D(o_de), D(o_gd), wg);
    if (want_grad)
      d3k::chain_kernel<<<nb, tb, 0, s>>>(total, n_mol, I(o_offs), I(o_set), dz, dxyz, D(o_de), D(o_gd), D(o_g));
    d3k::energy_kernel<<<(n_mol + tb - 1) / tb, tb, 0, s>>>(n_mol, I(o_offs), I(o_set), D(o_e6), D(o_e8), D(o_en));
    c->launches += want_grad ? 4 : 3;
  }
  if (nh) {
    h4k::Scratch S;
    S.V = D(o_s[0]);
    S.Hs = D(o_s[1]);
    S.Os = D(o_s[2]);
    S.sw = D(o_s[3]);
    S.swH = D(o_s[4]);
    S.swO = D(o_s[5]);
    S.chd = D(o_s[6]);
    S.chdV = D(o_s[7]);
    S.cha = D(o_s[8]);
    S.chaO1 = D(o_s[9]);
    S.chaCC = D(o_s[10]);
    S.chaO2 = D(o_s[11]);
    S.cc = I(o_s[12]);
    S.o2 = I(o_s[12]) + A;  // two int arrays share one double-sized slot
    S.adjH = D(o_s[13]);
    S.adjO = D(o_s[14]);
    S.adjV = D(o_s[15]);
    S.gB = D(o_gh);
    h4k::h4_kernel<<<nh, h4k::kThreads, 0, s>>>(I(o_hm), I(o_offs), I(o_var), dz, dxyz, S, D(o_eh), D(o_ho));
    ++c->launches;
  }
  if (nm) {
    CUDA_TRY(c, cudaMemsetAsync(D(o_mg), 0, 24 * A, s));
    mmk::mmok_kernel<<<nm, 128, 0, s>>>(I(o_mm), I(o_offs), dz, dxyz, D(o_me), D(o_mg));
    ++c->launches;
  }
  CUDA_TRY(c, cudaGetLastError());
  if (any_d3) {
    CUDA_TRY(c, cudaMemcpyAsync(hb + P.h_e, D(o_en), 8 * M, cudaMemcpyDeviceToHost, s));
    if (want_grad) CUDA_TRY(c, cudaMemcpyAsync(hb + P.h_gd3, D(o_g), 24 * A, cudaMemcpyDeviceToHost, s));
  }
  if (nh) {
    CUDA_TRY(c, cudaMemcpyAsync(hb + P.h_eh, D(o_eh), 24 * M, cudaMemcpyDeviceToHost, s));
    if (want_grad) CUDA_TRY(c, cudaMemcpyAsync(hb + P.h_gh, D(o_ho), 24 * A, cudaMemcpyDeviceToHost, s));
  }
  if (nm) {
    CUDA_TRY(c, cudaMemcpyAsync(hb + P.h_em, D(o_me), 8 * M, cudaMemcpyDeviceToHost, s));
    if (want_grad) CUDA_TRY(c, cudaMemcpyAsync(hb + P.h_gm, D(o_mg), 24 * A, cudaMemcpyDeviceToHost, s));
  }
  c->h2d += (long long)in_bytes;
  return PM3GPU_OK;
}

// After the stream has been synchronised: parts[5 m + {0,1,2,3,4}] = (D3, H4, H-H, X, MMOK) in eV for
// the molecules with any term, grad (optional, 3 per atom) the gradient of their sum in eV/Bohr for
// those molecules' atoms.
void corrections_collect(pm3gpu_ctx* c, const int32_t* h_offs, const CorrPlan& P, double* parts, double* grad) {
  if (!P.any) return;
  const char* hb = static_cast<const char*>(c->h_corr);
  const double* e = reinterpret_cast<const double*>(hb + P.h_e);
  const double* eh = reinterpret_cast<const double*>(hb + P.h_eh);
  const double* em = reinterpret_cast<const double*>(hb + P.h_em);
  const double* gd3 = reinterpret_cast<const double*>(hb + P.h_gd3);
  const double* gh = reinterpret_cast<const double*>(hb + P.h_gh);
  const double* gm = reinterpret_cast<const double*>(hb + P.h_gm);
  for (int m = 0; m < P.n_mol; ++m) {
    if (!P.set[m] && !P.is_h[m] && !P.is_m[m]) continue;
    double* p = parts + 5 * (size_t)m;
    p[0] = P.set[m] ? e[m] : 0.0;
    p[1] = P.is_h[m] ? eh[3 * m] : 0.0;
    p[2] = P.is_h[m] ? eh[3 * m + 1] : 0.0;
    p[3] = P.is_h[m] ? eh[3 * m + 2] : 0.0;
    p[4] = P.is_m[m] ? em[m] : 0.0;
    if (grad && P.grad)
      for (size_t k = 3 * (size_t)h_offs[m]; k < 3 * (size_t)h_offs[m + 1]; ++k)
        grad[k] = (P.set[m] ? gd3[k] : 0.0) + (P.is_h[m] ? gh[k] : 0.0) + (P.is_m[m] ? gm[k] : 0.0);
  }
}

// Launch, synchronise and collect: the correction-only entry points.
int corrections_batch(pm3gpu_ctx* c, int n_mol, const int32_t* h_offs, const int32_t* h_set, const int32_t* h_var,
                      const int32_t* h_mmok, const int32_t* dz, const double* dxyz, double* parts, double* grad) {
  CorrPlan P;
  const int rc = corrections_launch(c, n_mol, h_offs, h_set, h_var, h_mmok, dz, dxyz, grad != nullptr, P);
  if (rc != PM3GPU_OK) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  corrections_collect(c, h_offs, P, parts, grad);
  return PM3GPU_OK;
}

// The corrections each molecule's options ask for (variant, MMOK), launched ahead of the SCF.
int corrections_for_batch(pm3gpu_ctx* c, int n_mol, const int32_t* h_offs, const pm3gpu_options* opts, int per_mol,
                          const int32_t* dz, const double* dxyz, bool want_grad, CorrPlan& P) {
  std::vector<int32_t> var(n_mol, 0), set(n_mol, 0), mm(n_mol, 0);
  bool any = false;
  for (int m = 0; m < n_mol; ++m) {
    const pm3gpu_options* o = per_mol ? opts + m : opts;
    if (h_offs[m + 1] <= h_offs[m]) continue;
    if (o->variant >= PM3GPU_VARIANT_D3 && o->variant <= PM3GPU_VARIANT_D3H4X) {
      var[m] = o->variant;
      set[m] = o->variant == PM3GPU_VARIANT_D3 ? 1 : 2;  // the D3H4 family refits D3 (mod.rs:142-156)
      any = true;
    }
    if (o->mmok) {
      mm[m] = 1;
      any = true;
    }
  }
  P = CorrPlan{};
  if (!any) return PM3GPU_OK;
  return corrections_launch(c, n_mol, h_offs, set.data(), var.data(), mm.data(), dz, dxyz, want_grad, P);
}

// For the molecules that converged, the correction launched for them (corrections_for_batch) joins
// total_ev, the heat of formation and (when asked for) the gradient. The stream must be synchronised.
void apply_corrections(pm3gpu_ctx* c, int n_mol, const int32_t* h_offs, const int32_t* h_z, const CorrPlan& P,
                       pm3gpu_result* results, double* gradients) {
  if (!P.any) return;
  std::vector<double> parts(5 * (size_t)n_mol, 0.0), g(gradients && P.grad ? 3 * (size_t)h_offs[n_mol] : 0, 0.0);
  corrections_collect(c, h_offs, P, parts.data(), g.empty() ? nullptr : g.data());
  for (int m = 0; m < n_mol; ++m) {
    if (results[m].status != PM3GPU_OK || (!P.set[m] && !P.is_h[m] && !P.is_m[m])) continue;
    pm3gpu_result& R = results[m];
    double e_isol = 0.0, eheat = 0.0;
    for (int a = h_offs[m]; a < h_offs[m + 1]; ++a) {
      e_isol += c->h_elem[h_z[a]].e_isol;
      eheat += c->h_elem[h_z[a]].eheat_ev;
    }
    const double* p = parts.data() + 5 * (size_t)m;
    // correction_energy_with_mmok (mod.rs:240-250): the variant's sum, then the amide term
    const double corr = P.is_m[m] ? (p[0] + p[1] + p[2] + p[3]) + p[4] : (p[0] + p[1] + p[2] + p[3]);
    R.total_ev = R.electronic_ev + R.core_ev + corr;
    R.heat_of_formation_kcal = (R.total_ev - e_isol + eheat) * kEvToKcal;
    if (!g.empty())
      for (size_t k = 3 * (size_t)h_offs[m]; k < 3 * (size_t)h_offs[m + 1]; ++k) gradients[k] += g[k];
  }
}
