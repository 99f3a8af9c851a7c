// ccp_batch.cpp -- batches of independent frames over one model.
//
// A batch owns `slots` contexts (each with its own device buffers and CUDA streams) and one
// host worker thread per slot for the duration of a call.  Frame f of a call runs on slot
// f % slots through the single-frame entry point, so up to `slots` frames are in flight on
// the GPU at once: the frames of a batch are independent, and a frame of 256 waters leaves
// most of the GPU idle (its dipole iteration is latency-bound).  Results are identical to
// separate single-frame calls.  The reference evaluates one configuration per call; this
// has no counterpart there.
//
// FS3, the costliest term of a frame, can be fused across the frames when they share one box
// length (option "fuse_fs3", off by default: beside one long FS3 launch every frame's
// Ewald/induction chain slows down, and 32 frames of 256 waters took 35.8 ms fused against
// 33.7 ms with FS3 per frame, 8 slots): the batch then packs every frame's molecules one
// frame after another and runs one neighbour search, one triple enumeration and one FS3
// launch for all of them on its own stream (batch_fs3_launch), while the slots evaluate the
// other terms; the FS3 forces, energies and parameter gradients are then added per frame
// (batch_fs3_finish).  The results equal the single-frame calls'.
#include <string>
#include <thread>
#include <vector>

#include "ccp_internal.h"

struct ccp_batch {
  std::vector<ccp_context *> ctx;
  int nm = 0;
  bool fuse_fs3 = false;
  ccp::BatchFs3 fs3;
};

namespace {

int fail(int code, const std::string &msg) {
  ccp::set_error(msg);
  return code;
}

const double *off(const double *p, size_t n) { return p ? p + n : nullptr; }
double *off(double *p, size_t n) { return p ? p + n : nullptr; }

}  // namespace

extern "C" {

int ccp_batch_create(const ccp_model *m, int nm, double box0, int slots, int device,
                     int precision, ccp_batch **out) {
  if (!m || !out || nm < 1 || slots < 1 || slots > 256)
    return fail(CCP_ERR_BAD_INPUT, "ccp_batch_create: bad argument (slots must be 1..256)");
  *out = nullptr;
  ccp_batch *b = new ccp_batch;
  b->nm = nm;
  for (int s = 0; s < slots; s++) {
    ccp_context *c = nullptr;
    const int r = ccp_context_create(m, nm, box0, device, precision, &c);
    if (r) {
      const std::string msg = ccp_last_error();
      ccp_batch_destroy(b);
      return fail(r, "ccp_batch_create: context " + std::to_string(s) + ": " + msg);
    }
    b->ctx.push_back(c);
  }
  *out = b;
  return CCP_OK;
}

int ccp_batch_destroy(ccp_batch *b) {
  if (!b) return CCP_ERR_BAD_INPUT;
  ccp::batch_fs3_free(b->fs3);
  for (ccp_context *c : b->ctx) ccp_context_destroy(c);
  delete b;
  return CCP_OK;
}

int ccp_batch_slots(const ccp_batch *b, int *slots) {
  if (!b || !slots) return CCP_ERR_BAD_INPUT;
  *slots = (int)b->ctx.size();
  return CCP_OK;
}

int ccp_batch_context(ccp_batch *b, int slot, ccp_context **ctx) {
  if (!b || !ctx || slot < 0 || slot >= (int)b->ctx.size()) return CCP_ERR_BAD_INPUT;
  *ctx = b->ctx[slot];
  return CCP_OK;
}

int ccp_batch_set_option(ccp_batch *b, const char *name, int value) {
  if (!b || !name) return CCP_ERR_BAD_INPUT;
  if (std::string(name) == "fuse_fs3") {
    b->fuse_fs3 = value != 0;
    return CCP_OK;
  }
  for (ccp_context *c : b->ctx) {
    const int r = ccp_context_set_option(c, name, value);
    if (r) return r;
  }
  return CCP_OK;
}

int ccp_batch_set_fs3_params(ccp_batch *b, const double *cs_sr, const double *cs_lr, int ncoef,
                             const double *bgr_sr, const double *bgr_lr) {
  if (!b) return CCP_ERR_BAD_INPUT;
  for (ccp_context *c : b->ctx) {
    const int r = ccp_context_set_fs3_params(c, cs_sr, cs_lr, ncoef, bgr_sr, bgr_lr);
    if (r) return r;
  }
  return CCP_OK;
}

int ccp_batch_terms_device(ccp_batch *b, unsigned terms, int nframes, const double *box,
                           const double *x, const double *y, const double *z, const double *xs,
                           const double *ys, const double *zs, int ld, ccp_energies *e,
                           double *fxs, double *fys, double *fzs, double *fxfs2, double *fyfs2,
                           double *fzfs2, double *fxfs3, double *fyfs3, double *fzfs3,
                           double *idmx, double *idmy, double *idmz, double *pgrad,
                           int pgrad_len) {
  if (!b || !box || !e || nframes < 0)
    return fail(CCP_ERR_BAD_INPUT, "ccp_batch_terms_device: null batch, box or energies");
  if (nframes == 0) return CCP_OK;
  const int slots = (int)b->ctx.size();
  const size_t nm = (size_t)b->nm, nsite = nm * (size_t)ld;
  int ncoef = 0;
  if (pgrad) {
    // the layout of one frame's gradient: dcs_sr, dcs_lr (ncoef each), dbgr_sr, dbgr_lr (867 each)
    ncoef = (pgrad_len - 2 * 3 * 289) / 2;
    if (ncoef < 1 || pgrad_len != 2 * ncoef + 2 * 3 * 289)
      return fail(CCP_ERR_BAD_INPUT, "ccp_batch_terms_device: pgrad_len is not 2 ncoef + 1734");
  }
  // FS3 of all frames in one launch set when they share one box length
  bool fused = b->fuse_fs3 && (terms & CCP_TERM_FS3) && nframes > 1 && x && y && z && xs && ys &&
               zs;
  for (int f = 1; fused && f < nframes; f++) fused = box[f] == box[0];
  int model_s3 = 0;
  if (fused) {
    ccp_context_get_option(b->ctx[0], "fs3_available", &model_s3);
    fused = model_s3 != 0;
  }
  unsigned rest = terms;
  if (fused) {
    const int r = ccp::batch_fs3_launch(b->ctx[0], b->fs3, nframes, box[0], x, y, z, xs, ys, zs,
                                        ld, pgrad != nullptr);
    if (r) return fail(r, std::string("ccp_batch_terms_device: fused FS3: ") + ccp_last_error());
    rest &= ~unsigned(CCP_TERM_FS3);
  }
  std::vector<int> status(nframes, CCP_OK);
  std::vector<std::string> msg(nframes);
  auto work = [&](int slot) {
    ccp_context *c = b->ctx[slot];
    for (int f = slot; f < nframes; f += slots) {
      const size_t o = (size_t)f * nm, os = (size_t)f * nsite;
      int r = ccp_terms_device(c, rest, off(x, o), off(y, o), off(z, o), off(xs, os), off(ys, os),
                               off(zs, os), ld, box[f], e + f, off(fxs, os), off(fys, os),
                               off(fzs, os), off(fxfs2, o), off(fyfs2, o), off(fzfs2, o),
                               off(fxfs3, o), off(fyfs3, o), off(fzfs3, o), off(idmx, os),
                               off(idmy, os), off(idmz, os));
      if (!r && pgrad && !fused) {
        double *g = pgrad + (size_t)f * pgrad_len;
        r = ccp_context_fs3_param_grad(c, g, g + ncoef, ncoef, g + 2 * ncoef,
                                       g + 2 * ncoef + 3 * 289);
      }
      if (r) {
        status[f] = r;
        msg[f] = ccp_last_error();
        return;  // this slot's later frames are not run
      }
    }
  };
  if (slots == 1 || nframes == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    const int nt = nframes < slots ? nframes : slots;
    for (int s = 0; s < nt; s++) th.emplace_back(work, s);
    for (std::thread &t : th) t.join();
  }
  int first_bad = -1;
  for (int f = 0; f < nframes && first_bad < 0; f++)
    if (status[f]) first_bad = f;
  if (fused) {
    // always completes the fused launch, so that no work of this call outlives it
    const int r = ccp::batch_fs3_finish(b->ctx[0], b->fs3, nframes, ld, e, fxs, fys, fzs, fxfs3,
                                        fyfs3, fzfs3, pgrad, pgrad_len);
    if (r && first_bad < 0)
      return fail(r, std::string("ccp_batch_terms_device: fused FS3: ") + ccp_last_error());
  }
  if (first_bad >= 0)
    return fail(status[first_bad], "frame " + std::to_string(first_bad) + ": " + msg[first_bad]);
  return CCP_OK;
}

}  // extern "C"
