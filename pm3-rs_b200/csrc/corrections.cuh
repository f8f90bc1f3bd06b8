// Host side of the post-SCF corrections (pm3-rs src/corrections/mod.rs:129-213): buffers and
// launches of the D3 kernels (d3.cuh) and the H4 / H-H / X kernel (h4.cuh), and their place in the
// single point (src/scf.rs:740-743: the correction joins total_ev and the heat of formation) and the
// gradient (src/gradient.rs:240-262, 324-357: its gradient joins the SCF gradient). Included by
// pm3gpu.cu inside its private namespace, before run_batch.
#pragma once

// Corrections of the batch in dz / dxyz (device): molecule m takes D3 with the parameter set
// h_set[m] (0 none, 1 D3Params::pm3_d3, 2 D3Params::pm3_d3h4), when h_var[m] is 2 or 3
// (PM3-D3H4, PM3-D3H4X) the H4 and H-H terms, 3 adding X, and when h_mmok[m] (optional) the MMOK
// amide term. parts[5 m + {0,1,2,3,4}] receive (D3, H4, H-H, X, MMOK) in eV for the molecules with
// any term, grad (optional, 3 per atom) the gradient of their sum in eV/Bohr for those molecules'
// atoms. One synchronisation of the stream.
int corrections_batch(pm3gpu_ctx* c, int n_mol, const int32_t* h_offs, const int32_t* h_set, const int32_t* h_var,
                      const int32_t* h_mmok, const int32_t* dz, const double* dxyz, double* parts, double* grad) {
  const int total = h_offs[n_mol];
  if (n_mol <= 0 || total <= 0) return PM3GPU_OK;
  std::vector<int32_t> set(h_set, h_set + n_mol), hmols, mmols;
  for (int m = 0; m < n_mol; ++m) {
    if (h_var[m] >= 2 && h_offs[m + 1] > h_offs[m]) hmols.push_back(m);
    if (h_mmok && h_mmok[m] && h_offs[m + 1] > h_offs[m]) mmols.push_back(m);
  }
  const int nh = (int)hmols.size(), nm = (int)mmols.size();
  CUDA_TRY(c, d3_ready(c->device));
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t A = (size_t)total, M = (size_t)n_mol;
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o += up(b);
    return at;
  };
  const size_t o_offs = take(4 * (M + 1)), o_set = take(4 * M), o_var = take(4 * M), o_hm = take(4 * (size_t)nh + 4);
  const size_t o_cn = take(8 * A), o_de = take(8 * A), o_e6 = take(8 * A), o_e8 = take(8 * A);
  const size_t o_gd = take(24 * A), o_g = take(24 * A), o_en = take(8 * M), o_eh = take(24 * M);
  const size_t o_gh = take(nh ? 24 * A : 0), o_ho = take(nh ? 24 * A : 0);
  const size_t o_mm = take(4 * (size_t)nm + 4), o_me = take(nm ? 8 * M : 0), o_mg = take(nm ? 24 * A : 0);
  size_t o_s[16];
  for (int k = 0; k < 16; ++k) o_s[k] = take(nh ? 8 * A : 0);
  const size_t bytes = o;
  CUDA_TRY(c, c->d3buf.ensure(bytes));
  char* base = c->d3buf.as<char>();
  auto I = [&](size_t off) { return reinterpret_cast<int32_t*>(base + off); };
  auto D = [&](size_t off) { return reinterpret_cast<double*>(base + off); };
  cudaStream_t s = c->stream;
  CUDA_TRY(c, cudaMemcpyAsync(I(o_offs), h_offs, 4 * (M + 1), cudaMemcpyHostToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(I(o_set), set.data(), 4 * M, cudaMemcpyHostToDevice, s));
  const int tb = 128, nb = (total + tb - 1) / tb;
  const int wg = grad ? 1 : 0;
  d3k::cn_kernel<<<nb, tb, 0, s>>>(total, n_mol, I(o_offs), I(o_set), dz, dxyz, D(o_cn));
  d3k::pair_kernel<<<nb, tb, 0, s>>>(total, n_mol, I(o_offs), I(o_set), dz, dxyz, D(o_cn), D(o_e6), D(o_e8), D(o_de),
                                     D(o_gd), wg);
  if (grad) d3k::chain_kernel<<<nb, tb, 0, s>>>(total, n_mol, I(o_offs), I(o_set), dz, dxyz, D(o_de), D(o_gd), D(o_g));
  d3k::energy_kernel<<<(n_mol + tb - 1) / tb, tb, 0, s>>>(n_mol, I(o_offs), I(o_set), D(o_e6), D(o_e8), D(o_en));
  c->launches += grad ? 4 : 3;
  if (nh) {
    CUDA_TRY(c, cudaMemcpyAsync(I(o_var), h_var, 4 * M, cudaMemcpyHostToDevice, s));
    CUDA_TRY(c, cudaMemcpyAsync(I(o_hm), hmols.data(), 4 * (size_t)nh, cudaMemcpyHostToDevice, s));
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
    CUDA_TRY(c, cudaMemcpyAsync(I(o_mm), mmols.data(), 4 * (size_t)nm, cudaMemcpyHostToDevice, s));
    CUDA_TRY(c, cudaMemsetAsync(D(o_mg), 0, 24 * A, s));
    mmk::mmok_kernel<<<nm, 128, 0, s>>>(I(o_mm), I(o_offs), dz, dxyz, D(o_me), D(o_mg));
    ++c->launches;
  }
  CUDA_TRY(c, cudaGetLastError());
  std::vector<double> e(M), eh(nh ? 3 * M : 0), gd3(grad ? 3 * A : 0), gh(grad && nh ? 3 * A : 0);
  std::vector<double> em(nm ? M : 0), gm(grad && nm ? 3 * A : 0);
  if (nm) {
    CUDA_TRY(c, cudaMemcpyAsync(em.data(), D(o_me), 8 * M, cudaMemcpyDeviceToHost, s));
    if (grad) CUDA_TRY(c, cudaMemcpyAsync(gm.data(), D(o_mg), 24 * A, cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(c, cudaMemcpyAsync(e.data(), D(o_en), 8 * M, cudaMemcpyDeviceToHost, s));
  if (grad) CUDA_TRY(c, cudaMemcpyAsync(gd3.data(), D(o_g), 24 * A, cudaMemcpyDeviceToHost, s));
  if (nh) {
    CUDA_TRY(c, cudaMemcpyAsync(eh.data(), D(o_eh), 24 * M, cudaMemcpyDeviceToHost, s));
    if (grad) CUDA_TRY(c, cudaMemcpyAsync(gh.data(), D(o_ho), 24 * A, cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(c, cudaStreamSynchronize(s));
  std::vector<char> is_h(M, 0), is_m(M, 0);
  for (int m : hmols) is_h[m] = 1;
  for (int m : mmols) is_m[m] = 1;
  for (int m = 0; m < n_mol; ++m) {
    if (!set[m] && !is_h[m] && !is_m[m]) continue;
    double* p = parts + 5 * (size_t)m;
    p[0] = set[m] ? e[m] : 0.0;
    p[1] = is_h[m] ? eh[3 * m] : 0.0;
    p[2] = is_h[m] ? eh[3 * m + 1] : 0.0;
    p[3] = is_h[m] ? eh[3 * m + 2] : 0.0;
    p[4] = is_m[m] ? em[m] : 0.0;
    if (grad)
      for (size_t k = 3 * (size_t)h_offs[m]; k < 3 * (size_t)h_offs[m + 1]; ++k)
        grad[k] = (set[m] ? gd3[k] : 0.0) + (is_h[m] ? gh[k] : 0.0) + (is_m[m] ? gm[k] : 0.0);
  }
  return PM3GPU_OK;
}

// For the molecules that converged, the correction of their variant joins total_ev, the heat of
// formation and (when asked for) the gradient.
int apply_corrections(pm3gpu_ctx* c, int n_mol, const int32_t* h_offs, const int32_t* h_z, const pm3gpu_options* opts,
                      int per_mol, const int32_t* dz, const double* dxyz, pm3gpu_result* results, double* gradients) {
  std::vector<int32_t> var(n_mol, 0), set(n_mol, 0), mm(n_mol, 0);
  bool any = false;
  for (int m = 0; m < n_mol; ++m) {
    const pm3gpu_options* o = per_mol ? opts + m : opts;
    if (results[m].status != PM3GPU_OK || h_offs[m + 1] == h_offs[m]) continue;
    if (o->variant != PM3GPU_VARIANT_PM3) {
      var[m] = o->variant;
      set[m] = o->variant == PM3GPU_VARIANT_D3 ? 1 : 2;  // the D3H4 family refits D3 (mod.rs:142-156)
      any = true;
    }
    if (o->mmok) {
      mm[m] = 1;
      any = true;
    }
  }
  if (!any) return PM3GPU_OK;
  std::vector<double> parts(5 * (size_t)n_mol, 0.0), g(gradients ? 3 * (size_t)h_offs[n_mol] : 0, 0.0);
  const int rc = corrections_batch(c, n_mol, h_offs, set.data(), var.data(), mm.data(), dz, dxyz, parts.data(),
                                   gradients ? g.data() : nullptr);
  if (rc != PM3GPU_OK) return rc;
  for (int m = 0; m < n_mol; ++m) {
    if (!var[m] && !mm[m]) continue;
    pm3gpu_result& R = results[m];
    double e_isol = 0.0, eheat = 0.0;
    for (int a = h_offs[m]; a < h_offs[m + 1]; ++a) {
      e_isol += c->h_elem[h_z[a]].e_isol;
      eheat += c->h_elem[h_z[a]].eheat_ev;
    }
    const double* p = parts.data() + 5 * (size_t)m;
    // correction_energy_with_mmok (mod.rs:240-250): the variant's sum, then the amide term
    const double corr = mm[m] ? (p[0] + p[1] + p[2] + p[3]) + p[4] : (p[0] + p[1] + p[2] + p[3]);
    R.total_ev = R.electronic_ev + R.core_ev + corr;
    R.heat_of_formation_kcal = (R.total_ev - e_isol + eheat) * kEvToKcal;
    if (gradients)
      for (size_t k = 3 * (size_t)h_offs[m]; k < 3 * (size_t)h_offs[m + 1]; ++k) gradients[k] += g[k];
  }
  return PM3GPU_OK;
}
