// lbm_ops_impl.cuh — the storage-typed work of a single domain (initial
// state, the pull and AA step loops, import and export), written once as
// templates and instantiated for one storage format per translation unit
// (lbm_ops_f32.cu, lbm_ops_f16.cu, lbm_ops_bf16.cu, lbm_ops_f64.cu), so that
// the kernels of the four formats compile in parallel.
#pragma once
#include "lbm_domain.cuh"
#include "lbm_quad.cuh"

namespace lbm {

template <class S>
int ops_tensor_maps(lbm_domain* d, int sm_count) {
  return domain_tensor_maps<S>(d, sm_count);
}

// k_init: pull form: arF_0 in lat[1], its collision in lat[0]; AA: arF_0 in
// the natural layout of lat[0], collided by the first step
template <class S>
int ops_launch_init(lbm_domain* d, cudaStream_t st) {
  const InitParams ip = init_params(d);
  return with_model<S>(d, [&](auto coll, auto les) -> int {
    // pull: arF_0 in lat[1], its collision in lat[0]; AA: arF_0 in the
    // natural layout of lat[0], collided by the first step
    const bool aa = d->opt.stream_mode == LBM_STREAM_AA;
    StepArgs<S> a = make_args<S>(d, nullptr, d->lat[aa ? 0 : 1], 0);
    a.den_out = d->den[0];
    a.ux_out = d->ux;
    a.uy_out = d->uy;
    a.uz_out = d->uz;
    const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
    k_init<S, decltype(coll)::value, decltype(les)::value>
        <<<gr, b, 0, st>>>(a, aa ? nullptr : (S*)d->lat[0], ip);
    CK(cudaGetLastError());
    return LBM_OK;
  });
}

template <class S>
int ops_run_pull(lbm_domain* d, int nsteps) {
  return with_model<S>(d, [&](auto coll, auto les) -> int {
    constexpr int C = decltype(coll)::value;
    constexpr bool L = decltype(les)::value;
    // one plain step (no side outputs unless requested)
    auto step_args = [&](long long k, bool den, bool vel, int cur) {
      StepArgs<S> a = make_args<S>(d, d->lat[cur], d->lat[cur ^ 1], k);
      if (den) a.den_out = d->den[k & 1];
      if (vel) {
        a.ux_out = d->ux;
        a.uy_out = d->uy;
        a.uz_out = d->uz;
      }
      return a;
    };
    int plain = nsteps > 2 ? nsteps - 2 : 0;  // the last two steps write rho / u
    // whole graph chunks of kGraphSteps plain steps
    if (plain >= 2 * kGraphSteps) {
      cudaGraphExec_t& g = d->chunk[d->cur];
      if (!g) {
        if (!d->capture) CK(cudaStreamCreateWithFlags(&d->capture, cudaStreamNonBlocking));
        CK(cudaStreamBeginCapture(d->capture, cudaStreamCaptureModeThreadLocal));
        int cur = d->cur;
        long long k = d->step;
        for (int i = 0; i < kGraphSteps; ++i) {
          ++k;
          launch_step<S, C, L>(d, step_args(k, false, false, cur), d->capture);
          cur ^= 1;
        }
        cudaGraph_t graph;
        CK(cudaStreamEndCapture(d->capture, &graph));
        cudaError_t e = cudaGraphInstantiate(&g, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess)
          return set_error(LBM_ERR_CUDA, "graph instantiation failed: %s",
                           cudaGetErrorString(e));
      }
      while (plain >= kGraphSteps) {
        CK(cudaGraphLaunch(g, d->stream));
        d->step += kGraphSteps;  // even: cur and plane parity unchanged
        plain -= kGraphSteps;
      }
    }
    const int rest = plain + (nsteps > 2 ? 2 : nsteps);
    for (int i = 0; i < rest; ++i) {
      const long long k = d->step + 1;
      launch_step<S, C, L>(d, step_args(k, i >= rest - 2, i == rest - 1, d->cur), d->stream);
      d->cur ^= 1;
      d->step = k;
    }
    d->post_direct = false;
    CK(cudaGetLastError());
    return LBM_OK;
  });
}

// nsteps AA steps (local and neighbour steps alternate with the layout),
// in graph chunks where possible; the last two steps write the rho of their
// input arF (the previous-step density of the residual), then k_aa_macro
// writes rho and u of the final arF.
// rho and u of the AA state after step d->step into den[step & 1] and u,
// from either layout; the face buffers are those of AA step s (k = s + 1)
template <class S>
int ops_aa_macro(lbm_domain* d) {
  StepArgs<S> m = make_args<S>(d, d->lat[0], d->lat[0], d->step + 1);
  m.den_out = d->den[d->step & 1];
  m.ux_out = d->ux;
  m.uy_out = d->uy;
  m.uz_out = d->uz;
  const int layout =
      d->cur ? kAASwapped : (d->post_direct ? kAANaturalComplete : kAANaturalPending);
  const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
  k_aa_macro<S><<<gr, b, 0, d->stream>>>(m, layout);
  CK(cudaGetLastError());
  return LBM_OK;
}

template <class S>
int ops_run_aa(lbm_domain* d, int nsteps) {
  return with_model<S>(d, [&](auto coll, auto les) -> int {
    constexpr int C = decltype(coll)::value;
    constexpr bool L = decltype(les)::value;
    const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
    auto args = [&](long long k, bool den, int neighbor) {
      return aa_args<S>(d, k, den, neighbor);
    };
    // paired / quad rows (16-bit): k_aa_words, one word of two / four nodes
    // per thread, except the first step after the initial state (a local
    // step, whose slots are all at the node: the per-node step over the
    // domain's rows)
    // quad rows (16-bit): k_aa_words, one word of four nodes per thread,
    // except the first step after the initial state (a local step, whose
    // slots are all at the node: the per-node step over quad rows)
    [[maybe_unused]] bool words = false;
    [[maybe_unused]] dim3 bw(1, 1, 1), gw(1, 1, 1), gn(1, 1, 1);
    if constexpr (kDev<S>) {
      if (d->g.rows != kRowsPlain) {
        if (!aa_words_apply(d->g))
          return set_error(LBM_ERR_INVALID, "AA domain rows without the word step");
        words = true;
        const int nw = d->g.px / 4;
        bw = block_of(nw);
        gw = dim3((nw + bw.x - 1) / bw.x, d->g.nz, d->g.ny);  // local step: every row
        // neighbour step: rows off the faces, then the face rows
        const int fz = (aa_face_rows(d->g) + d->g.nz - 3) / (d->g.nz - 2);
        gn = dim3(gw.x, d->g.nz - 2, d->g.ny - 2 + fz);
        // channels: the buffer of the x-face values (k_aa_xface_rules)
        if (d->g.casetype == CHANNEL && !d->xrule)
          CK(cudaMalloc(&d->xrule, (size_t)10 * d->g.ny * d->g.nz * sizeof(float)));
      }
    }
    [[maybe_unused]] const unsigned gx =
        (unsigned)((2 * (d->g.ny - 2) * (d->g.nz - 2) + 127) / 128);
    auto launch = [&](cudaStream_t st, const StepArgs<S>& a, int nb, int entry) {
      if constexpr (kDev<S>) {
        if (words) {
          if (entry != kAAFromInit) {
            StepArgs<S> aw = a;
            aw.xrule = d->xrule;
            if (aw.sr) {
              if (nb)
                k_aa_words<S, C, L, true, 1, 2><<<gn, bw, 0, st>>>(aw, entry);
              else
                k_aa_words<S, C, L, true, 0, 2><<<gw, bw, 0, st>>>(aw, entry);
            } else {
              if (nb)
                k_aa_words<S, C, L, false, 1, 2><<<gn, bw, 0, st>>>(aw, entry);
              else
                k_aa_words<S, C, L, false, 0, 2><<<gw, bw, 0, st>>>(aw, entry);
            }
          } else {
            k_aa_step<S, C, L, 0><<<gr, b, 0, st>>>(a, entry);
          }
          if (d->xrule) {
            // the next step's x-face values, from the face planes this step wrote
            StepArgs<S> fa = a;
            fa.prho_in = a.prho_out;
            fa.pu_in = a.pu_out;
            k_aa_xface_rules<S><<<gx, 128, 0, st>>>(fa, d->xrule);
          }
          return;
        }
      }
      if (nb)
        k_aa_step<S, C, L, 1><<<gr, b, 0, st>>>(a, entry);
      else
        k_aa_step<S, C, L, 0><<<gr, b, 0, st>>>(a, entry);
    };
    auto one = [&](bool den) {
      const long long k = d->step + 1;
      const int entry = d->aa_first ? kAAFromInit : (d->post_direct ? kAAComplete : kAAPending);
      launch(d->stream, args(k, den, d->cur), d->cur, entry);
      d->aa_first = false;
      d->post_direct = false;
      d->cur ^= 1;
      d->step = k;
    };
    int left = nsteps;
    // the first step from a complete natural layout (initial state, import)
    // has its own entry mode: never inside a graph
    if ((d->aa_first || d->post_direct) && left > 0) {
      one(left <= 2);
      --left;
    }
    int plain = left > 2 ? left - 2 : 0;
    if (plain >= 2 * kGraphSteps) {
      cudaGraphExec_t& g = d->chunk[d->cur];
      if (!g) {
        if (!d->capture) CK(cudaStreamCreateWithFlags(&d->capture, cudaStreamNonBlocking));
        CK(cudaStreamBeginCapture(d->capture, cudaStreamCaptureModeThreadLocal));
        int cur = d->cur;
        long long k = d->step;
        for (int i = 0; i < kGraphSteps; ++i) {
          ++k;
          launch(d->capture, args(k, false, cur), cur, kAAPending);
          cur ^= 1;
        }
        cudaGraph_t graph;
        CK(cudaStreamEndCapture(d->capture, &graph));
        cudaError_t e = cudaGraphInstantiate(&g, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess)
          return set_error(LBM_ERR_CUDA, "graph instantiation failed: %s",
                           cudaGetErrorString(e));
      }
      while (plain >= kGraphSteps) {
        CK(cudaGraphLaunch(g, d->stream));
        d->step += kGraphSteps;  // even: the layout is unchanged
        plain -= kGraphSteps;
        left -= kGraphSteps;
      }
    }
    while (left > 0) {
      one(left <= 2);
      --left;
    }
    return ops_aa_macro<S>(d);
  });
}

// k_import from d->staging (the AoS arF already on the device)
template <class S>
int ops_import(lbm_domain* d, int padded) {
  return with_model<S>(d, [&](auto coll, auto les) -> int {
    const bool aa = d->opt.stream_mode == LBM_STREAM_AA;
    StepArgs<S> a = make_args<S>(d, nullptr, d->lat[aa ? 0 : 1], 0);
    a.den_out = d->den[0];
    a.ux_out = d->ux;
    a.uy_out = d->uy;
    a.uz_out = d->uz;
    const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
    k_import<S, decltype(coll)::value, decltype(les)::value>
        <<<gr, b, 0, d->stream>>>(a, d->staging, padded, aa ? nullptr : (S*)d->lat[0]);
    CK(cudaGetLastError());
    return LBM_OK;
  });
}

// k_export into d->staging
template <class S>
int ops_export(lbm_domain* d, int padded) {
  const bool aa = d->opt.stream_mode == LBM_STREAM_AA;
  // AA: the face buffers of AA step s are those of make_args with k = s + 1
  StepArgs<S> a = make_args<S>(d, d->lat[aa ? 0 : d->cur ^ 1], nullptr, d->step + (aa ? 1 : 0));
  const int mode = aa ? (d->cur ? kExportAASwapped
                                : (d->post_direct ? kExportDirect : kExportAANaturalPending))
                      : (d->post_direct ? kExportDirect : kExportPull);
  const dim3 b = block_of(d->g.nx), gr = grid_of(d->g, b);
  k_export<S><<<gr, b, 0, d->stream>>>(a, d->staging, padded, mode);
  CK(cudaGetLastError());
  return LBM_OK;
}

template <class S>
StorageOps make_ops() {
  StorageOps o;
  o.tensor_maps = &ops_tensor_maps<S>;
  o.launch_init = &ops_launch_init<S>;
  o.run_pull = &ops_run_pull<S>;
  o.run_aa = &ops_run_aa<S>;
  o.import_staging = &ops_import<S>;
  o.export_staging = &ops_export<S>;
  o.aa_macro = &ops_aa_macro<S>;
  return o;
}

}  // namespace lbm
