// The Engine's loop over a batch of graphs (kernels in batch_kernels.cuh).
// Included by engine.cu inside namespace glv, after the Engine class.

int Engine::batch_level(Batch &b, const Level &L, const std::vector<int64_t> &voff) {
  b.voff = voff;
  int64_t *d_off, *d_out;
  const int G = b.G;
  TRY(alloc(&d_off, G + 1)); TRY(alloc(&d_out, G + 1));
  TRY(upload(s_, d_off, voff));
  LAUNCH(k_fill_gid, std::max(1, std::min(G, nsm_ * 16)), 256, 0, s_, G, d_off, b.gid);
  LAUNCH(k_gather_i64, grid_for(G + 1, 256, nsm_ * 4), 256, 0, s_, (int64_t)G + 1, d_off, L.ptr,
         d_out);
  std::vector<int64_t> rp(G + 1);
  CK(cudaMemcpyAsync(rp.data(), d_out, (G + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  b.gnnz.assign(G, 0);
  for (int g = 0; g < G; ++g) b.gnnz[g] = rp[g + 1] - rp[g];
  dfree(d_off); dfree(d_out);
  return GLV_OK;
}

// Sublevels for the graphs on stale colours only (the others are properly
// coloured: one sublevel); see Engine::sublevels.
int Engine::sublevels_batch(const Level &L, const Batch &b, int32_t **d_sub, int *nsub) {
  *d_sub = nullptr;
  *nsub = 1;
  std::vector<int64_t> ptr(L.nv + 1);
  CK(cudaMemcpyAsync(ptr.data(), L.ptr, (L.nv + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  std::vector<int32_t> col(L.nv);
  CK(cudaMemcpyAsync(col.data(), color_, L.nv * sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  std::vector<int32_t> sub(L.nv, 0), tail;
  int mx = 0;
  for (int g = 0; g < b.G; ++g) {
    if (!b.stale[g] || !b.in_phase[g]) continue;
    const int64_t v0 = b.voff[g], v1 = b.voff[g + 1];
    if (v1 <= v0) continue;
    const int64_t e0 = ptr[v0], e1 = ptr[v1];
    tail.resize(std::max<int64_t>(e1 - e0, 1));
    if (e1 > e0)
      CK(cudaMemcpyAsync(tail.data(), L.tail + e0, (e1 - e0) * sizeof(int32_t),
                         cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    for (int64_t v = v0; v < v1; ++v) {
      int d = 0;
      for (int64_t j = ptr[v]; j < ptr[v + 1]; ++j) {
        const int32_t u = tail[j - e0];
        if (u < v && col[u] == col[v]) d = std::max(d, sub[u] + 1);
      }
      sub[v] = d;
      mx = std::max(mx, d);
    }
  }
  *nsub = mx + 1;
  if (mx == 0) return GLV_OK;
  TRY(alloc(d_sub, L.nv));
  CK(cudaMemcpyAsync(*d_sub, sub.data(), L.nv * sizeof(int32_t), cudaMemcpyHostToDevice, s_));
  CK(cudaStreamSynchronize(s_));
  return GLV_OK;
}

// The multiphase loop of Coloring/runMultiPhaseColoring.cpp:51-238 (and,
// with coloring off, BasicCommunitiesDetection/runMultiPhaseBasic.cpp:52-170)
// for every graph of a batch at once.  L0: the batch's level 0 (graph g owns
// [voff0[g], voff0[g+1])); d_C_orig: per original vertex, the final community
// in graph-local ids.
int Engine::run_multiphase_batch(const Level &L0, const std::vector<int64_t> &voff0,
                                 int32_t *d_C_orig, bool coloring, long min_graph_size,
                                 double threshold, double c_threshold, BatchResult *res) {
  if (ordered())
    return fail(GLV_ERR_UNSUPPORTED, "a batch in verify mode needs integral edge weights");
  const int G = (int)voff0.size() - 1;
  const double t_start = now_s();
  Batch b;
  b.G = G;
  TRY(alloc(&b.gid, nv0_ + 1));
  TRY(alloc(&b.gcst, G)); TRY(alloc(&b.gsum, G)); TRY(alloc(&b.gacc, 2 * G));
  TRY(alloc(&b.act, G));
  b.h_act.assign(G, 0); b.in_phase.assign(G, 0); b.stale.assign(G, 0);
  b.h_gcst.assign(G, 0.0); b.h_acc.assign(2 * G, 0.0); b.lower.assign(G, -1.0);
  b.mod.assign(G, 0.0); b.itr.assign(G, 0); b.done_s.assign(G, 0.0);
  // original vertices -> graph (for composing C_orig)
  int32_t *gid_orig, *cl_end, *d_cl_off, *Csave = nullptr;
  int64_t *d_orig_off, *d_lvl_off, *d_new_off;
  uint8_t *d_flag1, *d_flag2, *d_kind;
  TRY(alloc(&gid_orig, nv0_ + 1)); TRY(alloc(&cl_end, G)); TRY(alloc(&d_cl_off, G));
  TRY(alloc(&d_orig_off, G + 1)); TRY(alloc(&d_lvl_off, G + 1)); TRY(alloc(&d_new_off, G + 1));
  TRY(alloc(&d_flag1, G)); TRY(alloc(&d_flag2, G)); TRY(alloc(&d_kind, G));
  TRY(upload(s_, d_orig_off, voff0));
  LAUNCH(k_fill_gid, std::max(1, std::min(G, nsm_ * 16)), 256, 0, s_, G, d_orig_off, gid_orig);
  Level L = L0;
  L.owned = false;
  TRY(batch_level(b, L, voff0));
  bt_ = &b;
  struct GState {
    double prev = -1, curr = -1;
    long phase = 1;
    bool non_color = false, done = false;
    int tot_itr = 0;
    int64_t ncl = 0;
  };
  std::vector<GState> gs(G);
  for (auto &x : gs) x.non_color = !coloring;
  const long itr_cap = coloring ? 10000 : 100000;
  int ncolors = 0;
  double tcol = 0;
  if (coloring) {
    TRY(color(L, &ncolors, &tcol));
    t_color += tcol;
  }
  int rounds = 0;
  std::vector<uint8_t> cg(G), jg(G), kind(G), how(G);
  std::vector<int> itr_g(G);
  while (true) {
    ++rounds;
    bool any_c = false, any_j = false;
    for (int g = 0; g < G; ++g) {
      cg[g] = jg[g] = 0;
      itr_g[g] = 0;
      if (gs[g].done) continue;
      gs[g].prev = gs[g].curr;
      if (gs[g].non_color) { jg[g] = 1; any_j = true; }
      else { cg[g] = 1; any_c = true; }
    }
    double dm = 0;
    int di = 0;
    if (any_c) {
      b.in_phase = cg;
      bool stale_any = false;
      for (int g = 0; g < G; ++g) {
        b.lower[g] = gs[g].curr;
        stale_any = stale_any || (cg[g] && b.stale[g]);
      }
      b.thresh = c_threshold;
      TRY(coloring_phase(L, ncolors, stale_any, 0.0, c_threshold, &dm, &di));
      for (int g = 0; g < G; ++g)
        if (cg[g]) { gs[g].curr = b.mod[g]; itr_g[g] = b.itr[g]; }
      if (any_j) {
        TRY(alloc(&Csave, L.nv));
        CK(cudaMemcpyAsync(Csave, C, L.nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, s_));
      }
    }
    if (any_j) {
      b.in_phase = jg;
      for (int g = 0; g < G; ++g) b.lower[g] = gs[g].curr;
      b.thresh = threshold;
      TRY(basic_phase(L, 0.0, threshold, &dm, &di));
      for (int g = 0; g < G; ++g)
        if (jg[g]) { gs[g].curr = b.mod[g]; itr_g[g] = b.itr[g]; }
      if (any_c) {
        CK(cudaMemcpyAsync(d_flag1, cg.data(), G, cudaMemcpyHostToDevice, s_));
        LAUNCH(k_merge_group, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, b.gid, d_flag1,
               Csave, C);
      }
      dfree(Csave);
    }
    const double tc0 = now_s();
    // renumber the whole level; graph g's clusters are [cl_off[g], cl_end[g])
    int64_t ncl_all = 0;
    TRY(renumber(C, L.nv, &ncl_all));
    CK(cudaMemsetAsync(cl_end, 0, G * sizeof(int32_t), s_));
    LAUNCH(k_graph_cluster_end, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, b.gid, C,
           cl_end);
    std::vector<int32_t> h_end(G), h_off(G);
    CK(cudaMemcpyAsync(h_end.data(), cl_end, G * sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    int32_t run = 0;
    for (int g = 0; g < G; ++g) {
      h_off[g] = run;
      if (cg[g] || jg[g]) gs[g].ncl = std::max(0, h_end[g] - run);
      run = std::max(run, h_end[g]);
    }
    // compose C_orig of the graphs that swept in this round
    std::vector<uint8_t> took(G), first(G);
    for (int g = 0; g < G; ++g) {
      took[g] = (cg[g] || jg[g]) ? 1 : 0;
      first[g] = gs[g].phase == 1 ? 1 : 0;
    }
    CK(cudaMemcpyAsync(d_flag1, took.data(), G, cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_flag2, first.data(), G, cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(d_cl_off, h_off.data(), G * sizeof(int32_t), cudaMemcpyHostToDevice, s_));
    TRY(upload(s_, d_lvl_off, b.voff));
    LAUNCH(k_compose_batch, grid_for(nv0_, 256, nsm_ * 16), 256, 0, s_, nv0_, gid_orig,
           d_orig_off, d_lvl_off, d_cl_off, d_flag1, d_flag2, C, d_C_orig);
    // the phase loop's tests, graph by graph
    bool any_next = false;
    std::vector<int64_t> new_off(G + 1, 0);
    for (int g = 0; g < G; ++g) {
      kind[g] = NEXT_DONE;
      how[g] = 0;
      if (!took[g]) { new_off[g + 1] = new_off[g]; continue; }
      GState &x = gs[g];
      x.tot_itr += itr_g[g];
      bool stop = (x.phase > 200) || (x.tot_itr > itr_cap);
      const int64_t lvl_n = b.voff[g + 1] - b.voff[g];
      if (!stop) {
        if ((x.curr - x.prev) > threshold) {
          kind[g] = NEXT_COARSEN;
          ++x.phase;
          if (coloring && !x.non_color) how[g] = (x.ncl > min_graph_size) ? 1 : 2;
        } else if (coloring && !x.non_color) {
          x.non_color = true;
          kind[g] = NEXT_SAME;
        } else {
          stop = true;
        }
      }
      if (stop) {
        x.done = true;
        if (res) {
          res->final_modularity[g] = x.prev;
          res->phases[g] = (int)x.phase;
          res->iterations[g] = x.tot_itr;
          res->clusters[g] = (long)x.ncl;
          res->done_s[g] = now_s() - t_start;
        }
      } else {
        any_next = true;
      }
      const int64_t n_next = kind[g] == NEXT_COARSEN ? x.ncl : (kind[g] == NEXT_SAME ? lvl_n : 0);
      new_off[g + 1] = new_off[g] + n_next;
    }
    if (!any_next) {
      t_coarsen += now_s() - tc0;
      break;
    }
    // next level: the coarse graphs of coarsening graphs, the same graph for
    // graphs switching to Jacobi phases, nothing for finished ones
    CK(cudaMemcpyAsync(d_kind, kind.data(), G, cudaMemcpyHostToDevice, s_));
    TRY(upload(s_, d_new_off, new_off));
    LAUNCH(k_next_ids, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, b.gid, d_kind, d_lvl_off,
           d_new_off, d_cl_off, C, Ctgt);
    Level nl;
    int64_t ne = 0;
    TRY(coarsen(L, Ctgt, new_off[G], &nl, &ne));
    t_coarsen += now_s() - tc0;
    // colours of the next level
    bool any_fresh = false, any_stale = false;
    for (int g = 0; g < G; ++g) {
      any_fresh = any_fresh || how[g] == 1;
      any_stale = any_stale || how[g] == 2;
      b.stale[g] = (how[g] == 2) ? 1 : 0;
    }
    int32_t *old_color = nullptr;
    if (any_stale) {
      TRY(alloc(&old_color, L.nv));
      CK(cudaMemcpyAsync(old_color, color_, L.nv * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                         s_));
    }
    const std::vector<int64_t> old_voff = b.voff;
    free_level(L);
    L = nl;
    TRY(batch_level(b, L, new_off));
    if (any_fresh) {
      TRY(color(L, &ncolors, &tcol));
      t_color += tcol;
    }
    if (any_fresh || any_stale) {
      CK(cudaMemcpyAsync(d_flag1, how.data(), G, cudaMemcpyHostToDevice, s_));
      TRY(upload(s_, d_lvl_off, old_voff));
      if (!old_color) TRY(alloc(&old_color, 1));
      LAUNCH(k_stale_colors, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, b.gid, d_flag1,
             d_new_off, d_lvl_off, old_color, color_);
      int32_t *maxc;
      TRY(alloc(&maxc, 1));
      CK(cudaMemsetAsync(maxc, 0xff, sizeof(int32_t), s_));
      LAUNCH(k_max_color, grid_for(L.nv, 256, nsm_ * 8), 256, 0, s_, L.nv, color_, maxc);
      int32_t hm = -1;
      CK(cudaMemcpyAsync(&hm, maxc, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
      CK(cudaStreamSynchronize(s_));
      dfree(maxc);
      ncolors = hm + 1;
    }
    dfree(old_color);
  }
  free_level(L);
  bt_ = nullptr;
  dfree(b.gid); dfree(b.gcst); dfree(b.gsum); dfree(b.gacc); dfree(b.act);
  dfree(gid_orig); dfree(cl_end); dfree(d_cl_off);
  dfree(d_orig_off); dfree(d_lvl_off); dfree(d_new_off);
  dfree(d_flag1); dfree(d_flag2); dfree(d_kind);
  if (res) res->rounds = rounds;
  return GLV_OK;
}
