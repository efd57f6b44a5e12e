// Jacobi2d chare state machine (included by jacobi2d.cu inside its
// anonymous namespace; uses JBlock, japp, jproxy and the helpers above it).
//
// State of a chare: `pass` exchanges done, `iter` sweeps done (buf[pass & 1]
// holds u_iter), `sent` = last pass whose boundary was sent, got[p] = halos
// received for the pass of parity p. A halo for pass k is unpacked into the
// ghost zone of buf[k & 1] as soon as it arrives: pass k-1 reads only
// buf[(k-1) & 1] and writes only the interior of buf[k & 1], and a neighbour
// can be at most one pass ahead, so early halos need no stash (halo_mode 0).
// halo_mode 1 tags halos with refnum = pass instead, which parks early ones
// in the runtime's stash as the reference's refnum pattern would. Every
// chare of a problem computes the same pass lengths (pass_len), so residual
// checks fall on pass boundaries everywhere.

// Control flow is never re-entrant: pump() runs only at the top of an entry
// method; apply_decision() and tree_try_forward() report "the chare was
// parked and may continue" to their caller instead of resuming it
// themselves, so the call depth stays fixed whatever the message order.

// All threads: record the decision of check m.check and pass it down the
// tree. Returns 1 when the chare was parked on a decision (the caller then
// runs pump()).
template <typename T>
__device__ int apply_decision(JBlock& c, const jac::chare_desc& d, const jac::decision_msg& m) {
  __shared__ int s_resume;
  if (threadIdx.x == 0) {
    if (m.check > c.decided) c.decided = m.check;
    if (m.stop && c.stop_check < 0) c.stop_check = m.check;
    c.res0 = m.res0;
    c.res_last = m.res;
    c.checks = m.check + 1;
    s_resume = c.waiting;
    c.waiting = 0;
  }
  __syncthreads();
  int resume = s_resume;
  __syncthreads();
  jac::decision_msg fwd = m;
  for (int k = 0; k < 2; k++) {
    if (d.child[k] >= 0) jproxy->invoke(d.child[k], EP_DECISION, &fwd, sizeof(fwd));
  }
  return resume;
}

// All threads: when this chare's partial and its children's are in, send
// the sum up (fixed order: own, child 0, child 1) or decide at the root.
// Thread 0 alone reads and writes the chare and builds the message; the
// others only see it through shared memory. Returns apply_decision()'s
// resume flag (0 when nothing was decided).
template <typename T>
__device__ int tree_try_forward(JBlock& c, const jac::chare_desc& d, int chk) {
  __shared__ int s_act;
  __shared__ jac::partial_msg s_pm;
  __shared__ jac::decision_msg s_dm;
  if (threadIdx.x == 0) {
    s_act = 0;
    bool complete = c.have_own && (d.child[0] < 0 || c.child_got[0]) &&
                    (d.child[1] < 0 || c.child_got[1]);
    if (complete) {
      double t = c.own;
      if (d.child[0] >= 0) t += c.child_val[0];
      if (d.child[1] >= 0) t += c.child_val[1];
      c.have_own = 0;
      c.child_got[0] = c.child_got[1] = 0;
      if (d.parent >= 0) {
        s_pm.check = chk;
        s_pm.slot = (d.rank - 1) % 2;
        s_pm.gen = c.gen;
        s_pm.pad = 0;
        s_pm.value = t;
        s_act = 1;
      } else {
        const jac::prob_desc& p = c.prob;
        double nrm = sqrt(t);
        s_dm.check = chk;
        s_dm.gen = c.gen;
        s_dm.pad = 0;
        s_dm.res0 = (chk == 0) ? nrm : c.res0;
        s_dm.res = nrm;
        s_dm.stop = (p.tol > 0.0) && (s_dm.res0 == 0.0 || nrm <= p.tol * s_dm.res0) ? 1 : 0;
        s_act = 2;
      }
    }
  }
  __syncthreads();
  int act = s_act;
  jac::partial_msg pm = s_pm;
  jac::decision_msg dm = s_dm;
  __syncthreads();
  if (act == 1) {
    jproxy->invoke(d.parent, EP_PARTIAL, &pm, sizeof(pm));
  } else if (act == 2) {
    return apply_decision<T>(c, d, dm);
  }
  return 0;
}

// All threads: one pass buf[pass&1] -> buf[(pass+1)&1], then the residual
// tree when the pass starts at a check.
template <typename T>
__device__ void advance(JBlock& c, const jac::chare_desc& d) {
  const jac::prob_desc& p = c.prob;
  int K = p.check_every;
  // read before thread 0 advances the chare below
  const bool resid = K > 0 && (c.iter % K == 0);
  const int chk = K > 0 ? c.iter / K : 0;
  const int L = pass_len(d, p, c.iter);
  double part = sweep_block<T>(d, c.cur, resid, L);
  if (threadIdx.x == 0) {
    c.got[c.pass & 1] = 0;
    c.gotx[c.pass & 1] = 0;
    c.cur ^= 1;
    c.pass++;
    c.iter += L;
    if (resid) {
      c.own = part;
      c.have_own = 1;
    }
  }
  __syncthreads();
  // A decision taken here (at the tree root) cannot find this chare parked:
  // it is sweeping. pump()'s loop re-examines the state anyway.
  if (resid) tree_try_forward<T>(c, d, chk);
}

// All threads: drive the chare as far as it can go without new messages:
// decide (stop / park on a residual decision / continue), send the boundary
// of u_iter once, and sweep whenever all halos of the current sweep are in.
template <typename T>
__device__ void pump(JBlock& c, const jac::chare_desc& d) {
  const jac::prob_desc& p = c.prob;
  __shared__ int s_act;
  enum { IDLE = 0, SEND = 1, FIN = 2, SWEEP = 3, SELF = 4, SEND_Y = 5 };
  // lattice updates a chare without neighbours may run in one entry method
  // (a message round trip costs about as much as 20 K of them)
  long long self_budget = 1ll << 18;
  while (true) {
    if (threadIdx.x == 0) {
      int act = IDLE;
      int K = p.check_every;
      (void)CHARM_VERIFY(c.cur == (c.pass & 1) && c.got[0] <= c.nbr_count && c.got[1] <= c.nbr_count,
                   CHARMING_ERR_APP, 7000 + c.pass, c.i);
      if (c.done || c.waiting) {
        act = IDLE;
      } else if (c.sent < c.pass) {
        if (c.iter >= p.max_sweeps) {
          // finish only after the decision of the last residual check: the
          // result reports that check's norm, and no message of the problem
          // is left in flight (a serving worker can take the next request)
          if (K > 0 && p.max_sweeps > 0 && c.decided < (p.max_sweeps - 1) / K) {
            c.waiting = 1;
            act = IDLE;
          } else {
            act = FIN;
          }
        } else if (K > 0 && c.iter >= K && c.iter % K == 0 && c.decided < c.iter / K - 1) {
          c.waiting = 1;
          act = IDLE;
        } else if (K > 0 && c.iter >= K && c.iter % K == 0 && c.stop_check >= 0 &&
                   c.stop_check <= c.iter / K - 1) {
          act = FIN;
        } else {
          act = c.nbr_count > 0 ? SEND : SELF;
          c.sent = c.pass;
          if (act == SEND && japp::halo_mode() == 1) jproxy->set_refnum(c.i, c.pass);
        }
      } else if (d.ext > 0 && c.sent_y < c.pass && c.gotx[c.pass & 1] == c.nbx) {
        // two-phase: the left/right ghost columns of this pass are in, so
        // the top/bottom halos can carry the corners
        act = SEND_Y;
        c.sent_y = c.pass;
      } else if (c.nbr_count > 0 && c.got[c.pass & 1] == c.nbr_count && (d.ext == 0 || c.sent_y == c.pass)) {
        act = SWEEP;
      }
      s_act = act;
    }
    __syncthreads();
    int act = s_act;
    __syncthreads();
    if (act == IDLE) return;
    if (act == FIN) {
      finish(c, d);
      return;
    }
    if (act == SEND) {
      send_halos<T>(c, d, d.ext > 0 ? 1 : 0);
    } else if (act == SEND_Y) {
      send_halos<T>(c, d, 2);
    } else if (act == SELF) {
      // no neighbours: passes back to back up to a work budget, then one
      // message to itself, so other chares of the PE run in between
      if (self_budget > 0) {
        self_budget -= (long long)d.w * d.h * pass_len(d, p, c.iter);
        advance<T>(c, d);
        continue;
      }
      int it = c.pass;
      jproxy->invoke(c.i, EP_CONT, &it, sizeof(int));
      return;
    } else {
      advance<T>(c, d);
    }
  }
}

template <typename T>
__device__ void em_start_t(JBlock& c, void* arg) {
  if (japp::serving()) {
    // the start of a request travels down the residual tree
    const jac::start_msg m = *reinterpret_cast<const jac::start_msg*>(arg);
    if (!ensure_gen<T>(c, m.gen)) return;
    const jac::chare_desc& d = c.desc;
    for (int k = 0; k < 2; k++) {
      jac::start_msg f = m;
      if (d.child[k] >= 0) jproxy->invoke(d.child[k], EP_START, &f, sizeof(f));
    }
    pump<T>(c, d);
    return;
  }
  const jac::chare_desc& d = c.desc;
  if (threadIdx.x == 0) {
    count_nbrs(c, d);
    c.started = 1;
  }
  __syncthreads();
  pump<T>(c, d);
}

template <typename T>
__device__ void em_halo_t(JBlock& c, void* arg) {
  const jac::halo_hdr* hh = reinterpret_cast<const jac::halo_hdr*>(arg);
  if (!ensure_gen<T>(c, hh->gen)) return;
  if (c.done) return;
  const unsigned long long t_em = threadIdx.x == 0 ? pe_clock() : 0;
  const jac::chare_desc& d = c.desc;
  // checked build: direction, length and sweep of the halo are consistent
  if (!CHARM_VERIFY(hh->dir >= 0 && hh->dir < jac::N_DIRS && d.nbr[hh->dir] >= 0, CHARMING_ERR_APP,
                    1000 + hh->dir, c.i) ||
      !CHARM_VERIFY(hh->len == jac::halo_ghost(hh->dir, d).nr * jac::halo_ghost(hh->dir, d).nc,
                    CHARMING_ERR_APP, 2000 + hh->dir, hh->len) ||
      !CHARM_VERIFY(hh->pass == c.pass || hh->pass == c.pass + 1, CHARMING_ERR_APP,
                    3000 + (hh->pass - c.pass), c.i))
    return;
  unpack_halo<T>(c, d, arg);
  if (threadIdx.x == 0) {
    c.got[hh->pass & 1]++;
    if (hh->dir == jac::LEFT || hh->dir == jac::RIGHT) c.gotx[hh->pass & 1]++;
    (void)CHARM_VERIFY(c.got[hh->pass & 1] <= jac::N_DIRS, CHARMING_ERR_APP, 4000 + c.got[hh->pass & 1], c.i);
  }
  __syncthreads();
  if (threadIdx.x == 0) add_pe_cyc(2, pe_clock() - t_em);
  if (c.started) pump<T>(c, d);  // a halo may overtake the start message
}

template <typename T>
__device__ void em_cont_t(JBlock& c) {
  if (c.done) return;
  const jac::chare_desc& d = c.desc;
  advance<T>(c, d);
  pump<T>(c, d);
}

template <typename T>
__device__ void em_partial_t(JBlock& c, void* arg) {
  const jac::partial_msg* pm = reinterpret_cast<const jac::partial_msg*>(arg);
  if (!ensure_gen<T>(c, pm->gen)) return;
  if (c.done) return;
  const jac::chare_desc& d = c.desc;
  int chk = pm->check;
  // Thread 0 checks and records the partial; the others learn the outcome
  // after the barrier (reading child_got themselves would race with it).
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    bool ok = CHARM_VERIFY(pm->slot == 0 || pm->slot == 1, CHARMING_ERR_APP, 5000 + pm->slot, c.i) &&
              CHARM_VERIFY(d.child[pm->slot] >= 0 && !c.child_got[pm->slot], CHARMING_ERR_APP,
                           6000 + pm->slot, c.i);
    if (ok) {
      c.child_val[pm->slot] = pm->value;
      c.child_got[pm->slot] = 1;
    }
    s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  int ok = s_ok;
  __syncthreads();
  if (!ok) return;
  if (tree_try_forward<T>(c, d, chk)) pump<T>(c, d);
}

template <typename T>
__device__ void em_decision_t(JBlock& c, void* arg) {
  jac::decision_msg m = *reinterpret_cast<const jac::decision_msg*>(arg);
  if (!ensure_gen<T>(c, m.gen)) return;
  if (c.done) return;
  const jac::chare_desc& d = c.desc;
  __syncthreads();
  if (apply_decision<T>(c, d, m)) pump<T>(c, d);
}
