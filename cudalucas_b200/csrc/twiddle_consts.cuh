// e^{+2 pi i e / R} for the composite radices (80-bit precision, rounded once).
// Generated constants; e is a compile-time value after unrolling.
#pragma once
#include <cuda_runtime.h>
namespace llb {
template <int R> __device__ __forceinline__ double2 wconst(int e);
template <> __device__ __forceinline__ double2 wconst<6>(int e) {
  switch (((e % 6) + 6) % 6) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.5, 0.8660254037844386);
    case 2: return make_double2(-0.5, 0.8660254037844386);
    case 3: return make_double2(-1.0, 0.0);
    case 4: return make_double2(-0.5, -0.8660254037844386);
    case 5: return make_double2(0.5, -0.8660254037844386);
  }
  return make_double2(1.0, 0.0);
}
template <> __device__ __forceinline__ double2 wconst<9>(int e) {
  switch (((e % 9) + 9) % 9) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.766044443118978, 0.6427876096865394);
    case 2: return make_double2(0.17364817766693036, 0.984807753012208);
    case 3: return make_double2(-0.5, 0.8660254037844386);
    case 4: return make_double2(-0.9396926207859084, 0.3420201433256687);
    case 5: return make_double2(-0.9396926207859084, -0.3420201433256687);
    case 6: return make_double2(-0.5, -0.8660254037844386);
    case 7: return make_double2(0.17364817766693036, -0.984807753012208);
    case 8: return make_double2(0.766044443118978, -0.6427876096865394);
  }
  return make_double2(1.0, 0.0);
}
template <> __device__ __forceinline__ double2 wconst<10>(int e) {
  switch (((e % 10) + 10) % 10) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.8090169943749475, 0.5877852522924731);
    case 2: return make_double2(0.30901699437494745, 0.9510565162951535);
    case 3: return make_double2(-0.30901699437494745, 0.9510565162951535);
    case 4: return make_double2(-0.8090169943749475, 0.5877852522924731);
    case 5: return make_double2(-1.0, 0.0);
    case 6: return make_double2(-0.8090169943749475, -0.5877852522924731);
    case 7: return make_double2(-0.30901699437494745, -0.9510565162951535);
    case 8: return make_double2(0.30901699437494745, -0.9510565162951535);
    case 9: return make_double2(0.8090169943749475, -0.5877852522924731);
  }
  return make_double2(1.0, 0.0);
}
template <> __device__ __forceinline__ double2 wconst<12>(int e) {
  switch (((e % 12) + 12) % 12) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.8660254037844386, 0.5);
    case 2: return make_double2(0.5, 0.8660254037844386);
    case 3: return make_double2(0.0, 1.0);
    case 4: return make_double2(-0.5, 0.8660254037844386);
    case 5: return make_double2(-0.8660254037844386, 0.5);
    case 6: return make_double2(-1.0, 0.0);
    case 7: return make_double2(-0.8660254037844386, -0.5);
    case 8: return make_double2(-0.5, -0.8660254037844386);
    case 9: return make_double2(0.0, -1.0);
    case 10: return make_double2(0.5, -0.8660254037844386);
    case 11: return make_double2(0.8660254037844386, -0.5);
  }
  return make_double2(1.0, 0.0);
}
template <> __device__ __forceinline__ double2 wconst<14>(int e) {
  switch (((e % 14) + 14) % 14) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.9009688679024191, 0.4338837391175581);
    case 2: return make_double2(0.6234898018587335, 0.7818314824680298);
    case 3: return make_double2(0.2225209339563144, 0.9749279121818236);
    case 4: return make_double2(-0.2225209339563144, 0.9749279121818236);
    case 5: return make_double2(-0.6234898018587335, 0.7818314824680298);
    case 6: return make_double2(-0.9009688679024191, 0.4338837391175581);
    case 7: return make_double2(-1.0, 0.0);
    case 8: return make_double2(-0.9009688679024191, -0.4338837391175581);
    case 9: return make_double2(-0.6234898018587335, -0.7818314824680298);
    case 10: return make_double2(-0.2225209339563144, -0.9749279121818236);
    case 11: return make_double2(0.2225209339563144, -0.9749279121818236);
    case 12: return make_double2(0.6234898018587335, -0.7818314824680298);
    case 13: return make_double2(0.9009688679024191, -0.4338837391175581);
  }
  return make_double2(1.0, 0.0);
}
template <> __device__ __forceinline__ double2 wconst<20>(int e) {
  switch (((e % 20) + 20) % 20) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.9510565162951535, 0.30901699437494745);
    case 2: return make_double2(0.8090169943749475, 0.5877852522924731);
    case 3: return make_double2(0.5877852522924731, 0.8090169943749475);
    case 4: return make_double2(0.30901699437494745, 0.9510565162951535);
    case 5: return make_double2(0.0, 1.0);
    case 6: return make_double2(-0.30901699437494745, 0.9510565162951535);
    case 7: return make_double2(-0.5877852522924731, 0.8090169943749475);
    case 8: return make_double2(-0.8090169943749475, 0.5877852522924731);
    case 9: return make_double2(-0.9510565162951535, 0.30901699437494745);
    case 10: return make_double2(-1.0, 0.0);
    case 11: return make_double2(-0.9510565162951535, -0.30901699437494745);
    case 12: return make_double2(-0.8090169943749475, -0.5877852522924731);
    case 13: return make_double2(-0.5877852522924731, -0.8090169943749475);
    case 14: return make_double2(-0.30901699437494745, -0.9510565162951535);
    case 15: return make_double2(0.0, -1.0);
    case 16: return make_double2(0.30901699437494745, -0.9510565162951535);
    case 17: return make_double2(0.5877852522924731, -0.8090169943749475);
    case 18: return make_double2(0.8090169943749475, -0.5877852522924731);
    case 19: return make_double2(0.9510565162951535, -0.30901699437494745);
  }
  return make_double2(1.0, 0.0);
}
}  // namespace llb
