/*
 * transpose.h — reference-compatible C++ API (drop-in for kaihsin/213transpose
 * include/transpose.h:3-19).  Link with lib/libinplacett.a (this project's
 * build) instead of the reference's library of the same name.
 *
 * Layout: d1 is the fastest axis; every d3 slice is a row-major d2 x d1 matrix
 * that is transposed in place to d1 x d2.
 *
 * Instantiated for int, long long, float, double (as the reference) and for the
 * 16-byte types int4, float4, longlong2, double2.  data may be plain device
 * memory or managed memory (managed memory is prefetched to the current device
 * first, as the reference does).  The call runs on the legacy default stream
 * and returns after the transpose has finished.  Failures throw
 * std::runtime_error (the reference exits the process instead).
 */
#pragma once

namespace inplace {

namespace c2r {

template <typename T> void transpose(T* data, int d1, int d2, int d3);

}

namespace r2c {

template <typename T> void transpose(T* data, int d1, int d2, int d3);

}

template <typename T> void transpose(T* data, int d1, int d2, int d3);

}
