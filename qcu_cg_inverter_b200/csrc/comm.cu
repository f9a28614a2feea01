// Domain decomposition along t: the communicator, slab contexts, the halo
// exchange of spinor fields and the global sums of the solver's reductions.
//
// The reference splits the lattice over an MPI process grid and moves
// boundary half-spinors through host memory (src/qcu_communicator.cu:
// 1033-1268; dot products summed with MPI_Allreduce, :1603-1623). Here the
// lattice is cut into t-slabs, one per rank (one process per GPU). Every
// parity block of every field of a slab context has two ghost slices behind
// its sites (Geom::gfwd, Geom::gbwd); the stencil's t hops across the slab's
// faces read them (neighbours() in qcu_common.cuh), and everything else of the
// kernels is unchanged. Because a time slice is a whole number of 32-site
// blocks, a slice of any field - every RHS, every chunk, and the 16-bit norms -
// is one contiguous byte range, so the exchange needs no packing kernel: the
// first and last slices go straight from the field into the neighbours' ghost
// slices (ncclSend / ncclRecv on the context's stream, into the receiver's
// own memory; or through pinned host memory for the host transport).
//
// The clover term needs links up to one slice beyond the slab; a slab
// context therefore keeps an extended context of the slab plus two slices on
// each side (two, so that its parity matches the global one), which ingests
// the gauge field (the slab's links and the neighbours' boundary slices) and
// builds the clover fields with the ordinary kernels; the slab's own slices
// of its links and clover are copied into the slab context, together with
// the backward ghost slice of the links.
#include <dlfcn.h>
#include <nccl.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <string>
#include <type_traits>

#include "../../include/qcu_b200.h"
#include "qcu_context.h"

struct qcu_comm_s {
  int nranks = 1, rank = 0, device = 0;
  bool host = false;
  ncclComm_t nccl = nullptr;
  qcu_exchange_fn xfn = nullptr;
  qcu_allreduce_fn rfn = nullptr;
  void* user = nullptr;
  qcu::PinnedBuf hsend_lo, hsend_hi, hrecv_lo, hrecv_hi, hsum;
};

namespace qcu {

// NCCL is resolved at run time, on first use, from the libnccl.so.2 already
// in the process (a framework such as torch loads its own; linking another
// build at load time would shadow it) or else from QCU_NCCL_LIB / the system's.
struct NcclApi {
  ncclResult_t (*GetUniqueId)(ncclUniqueId*);
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int);
  ncclResult_t (*CommDestroy)(ncclComm_t);
  ncclResult_t (*GroupStart)();
  ncclResult_t (*GroupEnd)();
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t);
  const char* (*GetErrorString)(ncclResult_t);
};
static NcclApi g_nccl;
static bool g_nccl_ok = false;
static std::mutex g_nccl_mu;

static int nccl_load() {
  std::lock_guard<std::mutex> lk(g_nccl_mu);
  if (g_nccl_ok) return QCU_SUCCESS;
  void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);  // the process's own, if any
  const char* env = getenv("QCU_NCCL_LIB");
  if (!h && env) h = dlopen(env, RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h) {
    set_error(QCU_ERR_UNSUPPORTED, "NCCL (libnccl.so.2) is not available");
    return QCU_ERR_UNSUPPORTED;
  }
  bool ok = true;
  auto get = [&](auto& fn, const char* name) {
    fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
    ok = ok && fn != nullptr;
  };
  get(g_nccl.GetUniqueId, "ncclGetUniqueId");
  get(g_nccl.CommInitRank, "ncclCommInitRank");
  get(g_nccl.CommDestroy, "ncclCommDestroy");
  get(g_nccl.GroupStart, "ncclGroupStart");
  get(g_nccl.GroupEnd, "ncclGroupEnd");
  get(g_nccl.Send, "ncclSend");
  get(g_nccl.Recv, "ncclRecv");
  get(g_nccl.AllReduce, "ncclAllReduce");
  get(g_nccl.GetErrorString, "ncclGetErrorString");
  if (!ok) {
    set_error(QCU_ERR_UNSUPPORTED, "libnccl.so.2 lacks a function this library calls");
    return QCU_ERR_UNSUPPORTED;
  }
  g_nccl_ok = true;
  return QCU_SUCCESS;
}

static int nccl_status(ncclResult_t r, const char* what) {
  if (r == ncclSuccess) return QCU_SUCCESS;
  set_error(QCU_ERR_CUDA, std::string(what) + ": " + (g_nccl_ok ? g_nccl.GetErrorString(r) : "NCCL error"));
  return QCU_ERR_CUDA;
}
#define QCU_CHECK_NCCL(expr)                                    \
  do {                                                          \
    ncclResult_t _r = (expr);                                   \
    if (_r != ncclSuccess) return ::qcu::nccl_status(_r, #expr); \
  } while (0)

// One contiguous piece of a face exchange: send_lo -> rank-1 (its recv_hi),
// send_hi -> rank+1 (its recv_lo); device pointers.
struct FaceSeg {
  const void *send_lo, *send_hi;
  void *recv_lo, *recv_hi;
  size_t bytes;
};

static int comm_exchange(qcu_comm c, const void* send_lo, const void* send_hi, void* recv_lo, void* recv_hi,
                         size_t bytes, cudaStream_t st);

// Several pieces in one exchange (a 16-bit field's words and norms): one NCCL
// group, so the transfers of all pieces go together
static int comm_exchange_segs(qcu_comm c, const FaceSeg* seg, int n, cudaStream_t st) {
  if (c->host) {
    for (int i = 0; i < n; i++)
      QCU_CHECK(comm_exchange(c, seg[i].send_lo, seg[i].send_hi, seg[i].recv_lo, seg[i].recv_hi, seg[i].bytes, st));
    return QCU_SUCCESS;
  }
  const int lo = (c->rank + c->nranks - 1) % c->nranks, hi = (c->rank + 1) % c->nranks;
  // the same order on every rank: with two ranks lo == hi and the pairs match
  // in issue order (my send_lo with the peer's recv_hi); one rank sends to itself
  QCU_CHECK_NCCL(g_nccl.GroupStart());
  ncclResult_t r = ncclSuccess;  // the group is closed even when an operation fails
  for (int i = 0; i < n && r == ncclSuccess; i++) {
    if (!seg[i].bytes) continue;
    r = g_nccl.Send(seg[i].send_lo, seg[i].bytes, ncclChar, lo, c->nccl, st);
    if (r == ncclSuccess) r = g_nccl.Recv(seg[i].recv_hi, seg[i].bytes, ncclChar, hi, c->nccl, st);
    if (r == ncclSuccess) r = g_nccl.Send(seg[i].send_hi, seg[i].bytes, ncclChar, hi, c->nccl, st);
    if (r == ncclSuccess) r = g_nccl.Recv(seg[i].recv_lo, seg[i].bytes, ncclChar, lo, c->nccl, st);
  }
  const ncclResult_t e = g_nccl.GroupEnd();
  if (r != ncclSuccess) return nccl_status(r, "ncclSend/ncclRecv");
  return nccl_status(e, "ncclGroupEnd");
}

static int comm_exchange(qcu_comm c, const void* send_lo, const void* send_hi, void* recv_lo, void* recv_hi,
                         size_t bytes, cudaStream_t st) {
  if (bytes == 0) return QCU_SUCCESS;
  if (c->host && c->nranks == 1) {  // the slab is the whole lattice: its own faces, periodically
    QCU_CHECK_CUDA(cudaMemcpyAsync(recv_hi, send_lo, bytes, cudaMemcpyDeviceToDevice, st));
    QCU_CHECK_CUDA(cudaMemcpyAsync(recv_lo, send_hi, bytes, cudaMemcpyDeviceToDevice, st));
    return QCU_SUCCESS;
  }
  if (!c->host) {
    const FaceSeg s{send_lo, send_hi, recv_lo, recv_hi, bytes};
    return comm_exchange_segs(c, &s, 1, st);
  }
  for (PinnedBuf* b : {&c->hsend_lo, &c->hsend_hi, &c->hrecv_lo, &c->hrecv_hi}) QCU_CHECK(b->ensure(bytes));
  QCU_CHECK_CUDA(cudaMemcpyAsync(c->hsend_lo.p, send_lo, bytes, cudaMemcpyDeviceToHost, st));
  QCU_CHECK_CUDA(cudaMemcpyAsync(c->hsend_hi.p, send_hi, bytes, cudaMemcpyDeviceToHost, st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  if (c->xfn(c->user, c->hsend_lo.p, c->hsend_hi.p, c->hrecv_lo.p, c->hrecv_hi.p, bytes) != 0) {
    set_error(QCU_ERR_CUDA, "host transport: exchange failed");
    return QCU_ERR_CUDA;
  }
  QCU_CHECK_CUDA(cudaMemcpyAsync(recv_lo, c->hrecv_lo.p, bytes, cudaMemcpyHostToDevice, st));
  QCU_CHECK_CUDA(cudaMemcpyAsync(recv_hi, c->hrecv_hi.p, bytes, cudaMemcpyHostToDevice, st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(st));  // the pinned buffers are reused by the next call
  return QCU_SUCCESS;
}

static int comm_sum(qcu_comm c, double* values, int n, cudaStream_t st) {
  if (n <= 0 || (c->host && c->nranks == 1)) return QCU_SUCCESS;
  if (!c->host) {
    QCU_CHECK_NCCL(g_nccl.AllReduce(values, values, (size_t)n, ncclDouble, ncclSum, c->nccl, st));
    return QCU_SUCCESS;
  }
  QCU_CHECK(c->hsum.ensure(sizeof(double) * n));
  QCU_CHECK_CUDA(cudaMemcpyAsync(c->hsum.p, values, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  if (c->rfn(c->user, c->hsum.as<double>(), n) != 0) {
    set_error(QCU_ERR_CUDA, "host transport: allreduce failed");
    return QCU_ERR_CUDA;
  }
  QCU_CHECK_CUDA(cudaMemcpyAsync(values, c->hsum.p, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  return QCU_SUCCESS;
}

static size_t chunk_bytes_per_site(int prec) {
  return prec == PREC_DOUBLE ? 12 * 16 : (prec == PREC_SINGLE ? 6 * 16 : 3 * 16);
}

int dd_exchange(qcu_context ctx, const CSpinorView& v, int prec, cudaStream_t st) {
  const Geom& g = ctx->g;
  if (!g.tdd) return QCU_SUCCESS;
  const size_t f = (size_t)g.st;  // sites of a slice
  const size_t per = chunk_bytes_per_site(prec) * v.nrhs;
  char* d = const_cast<char*>(static_cast<const char*>(v.data));
  FaceSeg seg[2];
  int n = 0;
  seg[n++] = FaceSeg{d, d + (g.Vh - f) * per, d + g.gbwd * per, d + g.gfwd * per, f * per};
  if (prec == PREC_HALF) {
    const size_t pn = sizeof(float) * v.nrhs;
    char* m = const_cast<char*>(reinterpret_cast<const char*>(v.norm));
    seg[n++] = FaceSeg{m, m + (g.Vh - f) * pn, m + g.gbwd * pn, m + g.gfwd * pn, f * pn};
  }
  if (ctx->comm->host && ctx->comm->nranks == 1) {
    for (int i = 0; i < n; i++)
      QCU_CHECK(comm_exchange(ctx->comm, seg[i].send_lo, seg[i].send_hi, seg[i].recv_lo, seg[i].recv_hi, seg[i].bytes,
                              st));
    return QCU_SUCCESS;
  }
  return comm_exchange_segs(ctx->comm, seg, n, st);
}

// the interior of a slab stencil beside the face exchange (1), or the
// exchange first and then the whole slab (0)
#ifndef QCU_DD_OVERLAP
#define QCU_DD_OVERLAP 1
#endif

int dd_stencil(qcu_context ctx, const DslashArgs& a, int prec, LaunchShape sh, cudaStream_t st,
               const std::function<cudaError_t(const DslashArgs&)>& launch) {
  if (!QCU_DD_OVERLAP) {
    QCU_CHECK(dd_exchange(ctx, a.in, prec, st));
    QCU_CHECK_CUDA(launch(a));
    return QCU_SUCCESS;
  }
  const Geom& g = ctx->g;
  const int f = g.st;
  const int rt = (a.nrhs + sh.Rb - 1) / sh.Rb;  // RHS tiles
  // pieces: the interior slices, then the first and the last slice
  const int lo[3] = {f, 0, g.Vh - f}, hi[3] = {g.Vh - f, f, g.Vh};
  int tiles[3], total_tiles = 0;
  for (int k = 0; k < 3; k++) {
    tiles[k] = hi[k] > lo[k] ? (hi[k] - lo[k] + sh.Sb - 1) / sh.Sb : 0;
    total_tiles += tiles[k];
  }
  DslashArgs p[3];
  for (int k = 0, off = 0; k < 3; k++) {
    p[k] = a;
    p[k].s_off = lo[k];
    p[k].s_lim = hi[k];
    p[k].tile_off = off;
    p[k].tile_total = total_tiles;
    p[k].block_total = total_tiles * rt;
    off += tiles[k];
  }
  QCU_CHECK_CUDA(cudaEventRecord(ctx->dd_ev[0], st));  // the input is complete
  if (tiles[0]) QCU_CHECK_CUDA(launch(p[0]));        // the interior needs no ghost slice
  QCU_CHECK_CUDA(cudaStreamWaitEvent(ctx->dd_stream, ctx->dd_ev[0], 0));
  QCU_CHECK(dd_exchange(ctx, a.in, prec, ctx->dd_stream));
  QCU_CHECK_CUDA(cudaEventRecord(ctx->dd_ev[1], ctx->dd_stream));
  QCU_CHECK_CUDA(cudaStreamWaitEvent(st, ctx->dd_ev[1], 0));
  for (int k = 1; k < 3; k++)
    if (tiles[k]) QCU_CHECK_CUDA(launch(p[k]));
  return QCU_SUCCESS;
}

int dd_sum(qcu_context ctx, double* values, int n, cudaStream_t st) {
  if (!ctx->g.tdd) return QCU_SUCCESS;
  return comm_sum(ctx->comm, values, n, st);
}

}  // namespace qcu

namespace qcu {

// rows x width bytes from src (row pitch sp) to dst (row pitch dp), on st
static int copy2d(void* dst, size_t dp, const void* src, size_t sp, size_t width, size_t rows, cudaStream_t st) {
  if (!width || !rows) return QCU_SUCCESS;
  QCU_CHECK_CUDA(cudaMemcpy2DAsync(dst, dp, src, sp, width, rows, cudaMemcpyDeviceToDevice, st));
  return QCU_SUCCESS;
}

// The extended slab's links, ingested from its AoS field, to the slab: for
// every link format and (direction, parity) block, the slab's sites (the
// extended slices 2 .. Lt+1) and its two ghost slices (the slices just
// outside, 1 and Lt+2).
static int dd_links_from_ext(qcu_context ctx, const void* ext_aos) {
  qcu_context e = ctx->ext;
  QCU_CHECK(ingest_gauge(e, ext_aos));
  // the extended slab's stream writes its fields; the slab's stream copies them
  QCU_CHECK_CUDA(cudaStreamSynchronize(e->stream));
  const Geom& g = ctx->g;
  const Geom& ge = e->g;
  const size_t f = (size_t)g.st;
  for (int fmt : {(int)PREC_DOUBLE, (int)PREC_SINGLE, (int)PREC_HALF, (int)LINK_SINGLE18}) {
    DevBuf& dst = fmt == PREC_DOUBLE ? ctx->gauge64 : fmt == PREC_SINGLE ? ctx->gauge32 : fmt == PREC_HALF ? ctx->gauge16
                                                                                                         : ctx->gauge18;
    const DevBuf& src = fmt == PREC_DOUBLE ? e->gauge64 : fmt == PREC_SINGLE ? e->gauge32 : fmt == PREC_HALF ? e->gauge16
                                                                                                           : e->gauge18;
    QCU_CHECK(dst.ensure(gauge_field_bytes(fmt, g.Vh_pad), ctx->stream));
    const size_t per = gauge_field_bytes(fmt, 1) / 8;  // bytes of one link
    const size_t dp = per * g.Vh_pad, sp = per * ge.Vh_pad;  // (direction, parity) block pitches
    char* d = dst.as<char>();
    const char* s = src.as<char>();
    QCU_CHECK(copy2d(d, dp, s + 2 * f * per, sp, per * g.Vh, 8, ctx->stream));
    QCU_CHECK(copy2d(d + g.gbwd * per, dp, s + f * per, sp, per * f, 8, ctx->stream));
    QCU_CHECK(copy2d(d + g.gfwd * per, dp, s + (g.Lt + 2) * f * per, sp, per * f, 8, ctx->stream));
  }
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->gauge_loaded = true;
  ctx->gauge_version++;
  for (auto& c : ctx->clover.csw) c = NAN;
  return QCU_SUCCESS;
}

int dd_ingest_gauge(qcu_context ctx, const void* gauge) {
  const Geom& g = ctx->g;
  const Geom& ge = ctx->ext->g;
  cudaStream_t st = ctx->stream;
  const size_t link = 9 * 16, f = (size_t)g.st;
  const size_t blk = link * g.Vh, eblk = link * ge.Vh;  // (direction, parity) block of the slab / extension
  const void* src = gauge;
  if (!is_device_ptr_on(gauge, ctx->device)) {
    QCU_CHECK(ctx->stage_in.ensure(8 * blk, st));
    QCU_CHECK_CUDA(cudaMemcpyAsync(ctx->stage_in.p, gauge, 8 * blk, cudaMemcpyDefault, st));
    src = ctx->stage_in.p;
  }
  DevBuf ext_aos, sbuf;
  const size_t two = 2 * f * link;  // two slices of one block
  QCU_CHECK(ext_aos.ensure(8 * eblk, st));
  QCU_CHECK(sbuf.ensure(4 * 8 * two, st));  // send lo, send hi, recv lo, recv hi
  char* x = ext_aos.as<char>();
  const char* l = static_cast<const char*>(src);
  char *slo = sbuf.as<char>(), *shi = slo + 8 * two, *rlo = shi + 8 * two, *rhi = rlo + 8 * two;
  QCU_CHECK(copy2d(x + two, eblk, l, blk, blk, 8, st));           // the slab: extended slices 2 .. Lt+1
  QCU_CHECK(copy2d(slo, two, l, blk, two, 8, st));                // its first two slices
  QCU_CHECK(copy2d(shi, two, l + blk - two, blk, two, 8, st));    // its last two
  QCU_CHECK(comm_exchange(ctx->comm, slo, shi, rlo, rhi, 8 * two, st));
  QCU_CHECK(copy2d(x, eblk, rlo, two, two, 8, st));               // rank-1's last two: slices 0, 1
  QCU_CHECK(copy2d(x + eblk - two, eblk, rhi, two, two, 8, st));  // rank+1's first two: Lt+2, Lt+3
  QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  return dd_links_from_ext(ctx, ext_aos.p);
}

int dd_generate_gauge(qcu_context ctx, uint64_t seed, double eps) {
  const Geom& ge = ctx->ext->g;
  DevBuf ext_aos;
  QCU_CHECK(ext_aos.ensure((size_t)8 * ge.Vh * 9 * 16, ctx->stream));
  QCU_CHECK_CUDA(launch_gauge_random_slab(ge, ctx->Lt_global, ctx->t0 - 2, seed, eps, ext_aos.p, ctx->stream));
  ctx->launches++;
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return dd_links_from_ext(ctx, ext_aos.p);
}

// The slab's slices of clover slot ext_slot of the extended slab into slot
// `slot` of the slab: A (FP64) and A^-1 in FP64, FP32 and 16-bit with its norms.
int dd_clover_from_ext(qcu_context ctx, int ext_slot, int slot) {
  qcu_context e = ctx->ext;
  const Geom& g = ctx->g;
  const Geom& ge = e->g;
  const CloverBank& S = e->clover;
  CloverBank& D = ctx->clover;
  const size_t f = (size_t)g.st;
  struct Part {
    const void* s;
    void* d;
    size_t sstride, dstride, per;  // slot strides, bytes per site of one parity block
    size_t soff, doff;             // offset of the parity blocks within a slot
  };
  const size_t n16 = 9 * 16;  // 16-bit clover words per site; the norms follow both parity blocks
  const Part parts[5] = {
      {S.A64.p, D.A64.p, S.b64, D.b64, 36 * 16, 0, 0},
      {S.Ainv64.p, D.Ainv64.p, S.b64, D.b64, 36 * 16, 0, 0},
      {S.Ainv32.p, D.Ainv32.p, S.b32, D.b32, 18 * 16, 0, 0},
      {S.Ainv16.p, D.Ainv16.p, S.b16, D.b16, n16, 0, 0},
      {S.Ainv16.p, D.Ainv16.p, S.b16, D.b16, sizeof(float), 2 * ge.Vh_pad * n16, 2 * (size_t)g.Vh_pad * n16},
  };
  for (const Part& p : parts) {
    const char* s = static_cast<const char*>(p.s) + p.sstride * ext_slot + p.soff;
    char* d = static_cast<char*>(p.d) + p.dstride * slot + p.doff;
    // both parity blocks: rows of the slab's sites, pitched by the blocks
    QCU_CHECK(copy2d(d, p.per * g.Vh_pad, s + 2 * f * p.per, p.per * ge.Vh_pad, p.per * g.Vh, 2, ctx->stream));
  }
  return QCU_SUCCESS;
}

}  // namespace qcu

using namespace qcu;

extern "C" int qcuSlabGeometry(const int lattice[4], int nranks, int rank, int out[6]) {
  clear_error();
  if (!lattice || !out || lattice[0] <= 0 || lattice[0] % 2 || lattice[1] <= 0 || lattice[2] <= 0 ||
      lattice[3] <= 0 || rank < 0 || rank >= nranks || !slab_ok(lattice, nranks)) {
    set_error(QCU_ERR_INVALID_ARG,
              "the lattice does not split into t-slabs: Lt/nranks must be even and Lx/2*Ly*Lz a multiple of 32");
    return QCU_ERR_INVALID_ARG;
  }
  const Geom g = make_geom_slab(lattice, nranks, rank);
  out[0] = rank * g.Lt;
  out[1] = g.Lt;
  out[2] = g.st;
  out[3] = g.Vh;
  out[4] = g.gfwd;
  out[5] = g.gbwd;
  return QCU_SUCCESS;
}

extern "C" int qcuCommNcclUniqueId(void* id, int bytes) {
  clear_error();
  if (!id || bytes < (int)sizeof(ncclUniqueId)) {
    set_error(QCU_ERR_INVALID_ARG, "the NCCL unique id needs 128 bytes");
    return QCU_ERR_INVALID_ARG;
  }
  QCU_CHECK(nccl_load());
  ncclUniqueId u;
  QCU_CHECK_NCCL(g_nccl.GetUniqueId(&u));
  memcpy(id, &u, sizeof(u));
  return QCU_SUCCESS;
}

extern "C" int qcuCommCreateNccl(qcu_comm* comm, const void* id, int nranks, int rank, int device) {
  clear_error();
  if (!comm || !id || nranks < 1 || rank < 0 || rank >= nranks) {
    set_error(QCU_ERR_INVALID_ARG, "bad communicator arguments");
    return QCU_ERR_INVALID_ARG;
  }
  QCU_CHECK(nccl_load());
  QCU_CHECK_CUDA(cudaSetDevice(device));
  qcu_comm c = new qcu_comm_s();
  c->nranks = nranks;
  c->rank = rank;
  c->device = device;
  ncclUniqueId u;
  memcpy(&u, id, sizeof(u));
  ncclResult_t r = g_nccl.CommInitRank(&c->nccl, nranks, u, rank);
  if (r != ncclSuccess) {
    delete c;
    return nccl_status(r, "ncclCommInitRank");
  }
  *comm = c;
  return QCU_SUCCESS;
}

extern "C" int qcuCommCreateHost(qcu_comm* comm, int nranks, int rank, qcu_exchange_fn exchange,
                                 qcu_allreduce_fn allreduce, void* user) {
  clear_error();
  if (!comm || nranks < 1 || rank < 0 || rank >= nranks || (nranks > 1 && (!exchange || !allreduce))) {
    set_error(QCU_ERR_INVALID_ARG, "bad communicator arguments");
    return QCU_ERR_INVALID_ARG;
  }
  qcu_comm c = new qcu_comm_s();
  c->nranks = nranks;
  c->rank = rank;
  c->host = true;
  c->xfn = exchange;
  c->rfn = allreduce;
  c->user = user;
  *comm = c;
  return QCU_SUCCESS;
}

extern "C" int qcuCommDestroy(qcu_comm comm) {
  clear_error();
  if (!comm) return QCU_SUCCESS;
  if (comm->nccl) g_nccl.CommDestroy(comm->nccl);
  delete comm;
  return QCU_SUCCESS;
}

extern "C" int qcuContextCreateSlab(qcu_context* out, const int lattice[4], qcu_comm comm, int device) {
  clear_error();
  int geo[6];
  if (!out || !comm) {
    set_error(QCU_ERR_INVALID_ARG, "null context or communicator");
    return QCU_ERR_INVALID_ARG;
  }
  QCU_CHECK(qcuSlabGeometry(lattice, comm->nranks, comm->rank, geo));
  if (!comm->host && device != comm->device) {
    set_error(QCU_ERR_INVALID_ARG, "the slab's device is not the communicator's");
    return QCU_ERR_INVALID_ARG;
  }
  const int local[4] = {lattice[0], lattice[1], lattice[2], geo[1]};
  const int extended[4] = {lattice[0], lattice[1], lattice[2], geo[1] + 4};
  qcu_context ctx = nullptr, ext = nullptr;
  QCU_CHECK(qcuContextCreate(&ctx, local, device));
  int st = qcuContextCreate(&ext, extended, device);
  if (st != QCU_SUCCESS) {
    qcuContextDestroy(ctx);
    return st;
  }
  ctx->g = make_geom_slab(lattice, comm->nranks, comm->rank);
  ctx->comm = comm;
  ctx->ext = ext;
  if (cudaStreamCreateWithFlags(&ctx->dd_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->dd_ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->dd_ev[1], cudaEventDisableTiming) != cudaSuccess) {
    const cudaError_t e = cudaGetLastError();
    qcuContextDestroy(ctx);
    return cuda_status(e, "slab exchange stream");
  }
  ctx->Lt_global = lattice[3];
  ctx->t0 = geo[0];
  *out = ctx;
  return QCU_SUCCESS;
}

namespace qcu {
// Solves on a slab may replay CUDA graphs unless the host transport (host
// callbacks and stream synchronisations inside every exchange) serves it.
bool dd_graphs_ok(qcu_context ctx) { return !ctx->comm || !ctx->comm->host; }
}  // namespace qcu
