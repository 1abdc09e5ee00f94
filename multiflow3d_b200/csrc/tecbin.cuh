// Restart files `tecbin<id>.bin` of the reference: the writer of
// post.for:496-548 and the reader of initial.for:689-760, with the record
// stream decoded and encoded on the device.
//
// File layout (gfortran unformatted sequential: every record framed by its
// length in bytes as a 4-byte integer before and after it; default 4-byte
// integers, 8-byte reals under -fdefault-real-8):
//   record 1: toti, totj, totk          (3 int32)
//   record 2: pl                        (int32)
//   record 3: inind, jnind, knind       (3 int32: -1 where the block ends on
//                                        a wall, post.for:519-523)
//   then toti*totj*totk records, k outermost, i fastest, each 19 doubles:
//     x(i), y(j), z(k), p, pm, ppm, vis, u, um, uum, v, vm, vvm, w, wm, wwm,
//     uvm, uwm, vwm
// so cell record r (160 bytes: 4 + 152 + 4) is element r of a ttc array.
// The data records start at byte 52, a 4-byte boundary: the kernels move
// 4-byte words, staging a CTA's records in shared memory so that both the
// file words and the 16 field arrays are read and written coalesced.
#pragma once

namespace mf3d {

constexpr int TB_FIELDS = 19;                 // doubles per cell record
constexpr int TB_PAYLOAD = TB_FIELDS * 8;     // 152 bytes
constexpr int TB_WORDS = TB_PAYLOAD / 4 + 2;  // 40 words per framed record
constexpr long long TB_DATA = 52;             // three framed header records
constexpr int TB_CTA = 128;                   // records per CTA
constexpr int TB_SW = TB_WORDS + 1;           // shared-memory pitch of a record (odd: no bank conflicts)

struct TbPtrs {  // the 16 field arrays, passed by value
  double *p[16];
};

__device__ int g_tecbin_err;  // first bad record + 1 (0: none)

// Decode: cell record r -> out[f][r] for the 16 fields the reader keeps
// (initial.for:718-733: p .. vwm, record fields 4..19); a null out[f] skips
// the field.  Every record's two length words are checked against 152.
__global__ void __launch_bounds__(TB_CTA) k_tecbin_decode(const unsigned *__restrict__ words, long long nrec,
                                                         TbPtrs out) {
  pdl_wait();
  __shared__ unsigned s[TB_CTA * TB_SW];
  const long long r0 = (long long)blockIdx.x * TB_CTA;
  const int nr = (int)min((long long)TB_CTA, nrec - r0);
  const unsigned *src = words + r0 * TB_WORDS;
  for (int w = threadIdx.x; w < nr * TB_WORDS; w += TB_CTA) {
    const int q = w / TB_WORDS;
    s[q * TB_SW + (w - q * TB_WORDS)] = src[w];
  }
  __syncthreads();
  if (threadIdx.x >= nr) return;
  const unsigned *rec = s + threadIdx.x * TB_SW;
  const long long r = r0 + threadIdx.x;
  if (rec[0] != TB_PAYLOAD || rec[TB_WORDS - 1] != TB_PAYLOAD) {
    atomicCAS(&g_tecbin_err, 0, (int)min(r + 1, (long long)0x7fffffff));
    return;
  }
  for (int f = 3; f < TB_FIELDS; ++f) {
    double *o = out.p[f - 3];
    if (!o) continue;
    const unsigned long long lo = rec[1 + 2 * f], hi = rec[2 + 2 * f];
    o[r] = __longlong_as_double((long long)(lo | (hi << 32)));
  }
}

// Encode: the writer's record per cell from the node coordinates x(i),
// y(j), z(k) and the 16 fields (a null field writes zeros).
__global__ void __launch_bounds__(TB_CTA) k_tecbin_encode(unsigned *__restrict__ words, int toti, int totj,
                                                         long long nrec, const double *__restrict__ x,
                                                         const double *__restrict__ y, const double *__restrict__ z,
                                                         TbPtrs in) {
  pdl_wait();
  __shared__ unsigned s[TB_CTA * TB_SW];
  const long long r0 = (long long)blockIdx.x * TB_CTA;
  const int nr = (int)min((long long)TB_CTA, nrec - r0);
  if (threadIdx.x < nr) {
    const long long r = r0 + threadIdx.x;
    const int i = (int)(r % toti), j = (int)((r / toti) % totj), k = (int)(r / ((long long)toti * totj));
    unsigned *rec = s + threadIdx.x * TB_SW;
    rec[0] = TB_PAYLOAD;
    rec[TB_WORDS - 1] = TB_PAYLOAD;
    for (int f = 0; f < TB_FIELDS; ++f) {
      const double v = f == 0 ? x[i] : f == 1 ? y[j] : f == 2 ? z[k] : (in.p[f - 3] ? in.p[f - 3][r] : 0.0);
      const unsigned long long b = (unsigned long long)__double_as_longlong(v);
      rec[1 + 2 * f] = (unsigned)(b & 0xffffffffull);
      rec[2 + 2 * f] = (unsigned)(b >> 32);
    }
  }
  __syncthreads();
  unsigned *dst = words + r0 * TB_WORDS;
  for (int w = threadIdx.x; w < nr * TB_WORDS; w += TB_CTA) {
    const int q = w / TB_WORDS;
    dst[w] = s[q * TB_SW + (w - q * TB_WORDS)];
  }
}

}  // namespace mf3d

extern "C" {

int mf3d_tecbin_info_of(const void *image, size_t nbytes, mf3d_tecbin_info *info) {
  using namespace mf3d;
  if (!image || !info) { set_error("mf3d_tecbin_info_of: bad arguments"); return MF3D_E_INVALID; }
  if (nbytes < (size_t)TB_DATA) { set_error("tecbin: shorter than its header records"); return MF3D_E_INVALID; }
  int w[13];
  std::memcpy(w, image, sizeof w);
  // three framed records: (12 | 3 ints | 12), (4 | int | 4), (12 | 3 ints | 12)
  if (w[0] != 12 || w[4] != 12 || w[5] != 4 || w[7] != 4 || w[8] != 12 || w[12] != 12) {
    set_error("tecbin: header records are not framed as the reference writes them");
    return MF3D_E_INVALID;
  }
  info->toti = w[1]; info->totj = w[2]; info->totk = w[3];
  info->pl = w[6];
  info->inind = w[9]; info->jnind = w[10]; info->knind = w[11];
  if (info->toti < 1 || info->totj < 1 || info->totk < 1) { set_error("tecbin: bad extents"); return MF3D_E_INVALID; }
  info->records = (long long)info->toti * info->totj * info->totk;
  info->data_offset = TB_DATA;
  if ((long long)nbytes != TB_DATA + info->records * TB_WORDS * 4) {
    set_error("tecbin: size does not match toti*totj*totk cell records of 19 doubles");
    return MF3D_E_INVALID;
  }
  return MF3D_OK;
}

long long mf3d_tecbin_size(int toti, int totj, int totk) {
  if (toti < 1 || totj < 1 || totk < 1) return -1;
  return mf3d::TB_DATA + (long long)toti * totj * totk * mf3d::TB_WORDS * 4;
}

int mf3d_tecbin_decode_device(const void *image, const mf3d_tecbin_info *info, double *const *out, int device) {
  using namespace mf3d;
  if (!image || !info || !out || info->records < 1) { set_error("mf3d_tecbin_decode_device: bad arguments"); return MF3D_E_INVALID; }
  CK(cudaSetDevice(device));
  TbPtrs ptrs;
  std::memcpy(ptrs.p, out, sizeof ptrs.p);
  const int zero = 0;
  CK(cudaMemcpyToSymbol(g_tecbin_err, &zero, sizeof zero));
  const long long nblk = (info->records + TB_CTA - 1) / TB_CTA;
  if (nblk > 0x7fffffffLL) { set_error("tecbin: too many records"); return MF3D_E_INVALID; }
  const unsigned *words = (const unsigned *)((const char *)image + info->data_offset);
  k_tecbin_decode<<<(unsigned)nblk, TB_CTA>>>(words, info->records, ptrs);
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { set_error(std::string("tecbin decode: ") + cudaGetErrorString(e)); return MF3D_E_CUDA; }
  int bad = 0;
  CK(cudaMemcpyFromSymbol(&bad, g_tecbin_err, sizeof bad));
  if (bad) {
    set_error("tecbin: cell record " + std::to_string(bad - 1) + " is not framed as 152 bytes");
    return MF3D_E_INVALID;
  }
  return MF3D_OK;
}

int mf3d_tecbin_encode_device(int toti, int totj, int totk, int pl, int inind, int jnind, int knind,
                              const double *x, const double *y, const double *z, const double *const *fields,
                              void *image, int device) {
  using namespace mf3d;
  if (!x || !y || !z || !fields || !image || toti < 1 || totj < 1 || totk < 1) {
    set_error("mf3d_tecbin_encode_device: bad arguments");
    return MF3D_E_INVALID;
  }
  CK(cudaSetDevice(device));
  const int head[13] = {12, toti, totj, totk, 12, 4, pl, 4, 12, inind, jnind, knind, 12};
  CK(cudaMemcpy(image, head, sizeof head, cudaMemcpyHostToDevice));
  const long long nrec = (long long)toti * totj * totk;
  const long long nblk = (nrec + TB_CTA - 1) / TB_CTA;
  if (nblk > 0x7fffffffLL) { set_error("tecbin: too many records"); return MF3D_E_INVALID; }
  TbPtrs ptrs;
  for (int f = 0; f < 16; ++f) ptrs.p[f] = const_cast<double *>(fields[f]);
  unsigned *words = (unsigned *)((char *)image + TB_DATA);
  k_tecbin_encode<<<(unsigned)nblk, TB_CTA>>>(words, toti, totj, nrec, x, y, z, ptrs);
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { set_error(std::string("tecbin encode: ") + cudaGetErrorString(e)); return MF3D_E_CUDA; }
  return MF3D_OK;
}

}  // extern "C"
