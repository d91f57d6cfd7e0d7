// halo_oracle.cpp -- CPU restatement of the halo pack/unpack kernels.
//
// TEST INFRASTRUCTURE ONLY (checker for the CUDA halo kernels).
//
// Follows src/OpenCL/Kernels/halo_exchange.cl:
//   exchange_N_halo_read  (:156-291)  -> pack   (outer ring -> buffer)
//   exchange_N_halo_write (:3-152)    -> unpack (buffer -> outer ring)
// and src/OpenCL/Kernels/halo_exchange_correct.cl:
//   read  -> pack_inner   (the owned inner ring, without corners in N|S)
//   write -> unpack_inner (north/south buffer index without the im*w term)
// Buffer order: north|south|west|east per vector component, components
// stacked with stride v_sz.  The array holds v_dim floats per point; element
// (idx, v) lives at a[idx*es + v*vs] so that both the kernels' AoS layout
// (es=v_dim, vs=1) and the reference's C test programs' SoA layout (es=1,
// vs=im*jm*km) can be expressed.
#include <cstddef>

namespace {

inline size_t vsz_outer(unsigned im, unsigned jm, unsigned km, unsigned hw) {
    return 2ull * km * im * hw + 2ull * km * (jm - 2 * hw) * hw;
}
inline size_t vsz_inner(unsigned im, unsigned jm, unsigned km, unsigned hw) {
    return 2ull * km * (im + jm - 4 * hw) * hw;
}

}  // namespace

extern "C" {

size_t oracle_halo_buffer_floats(unsigned im, unsigned jm, unsigned km, unsigned hw, unsigned vdim,
                                 int inner) {
    return (size_t)vdim * (inner ? vsz_inner(im, jm, km, hw) : vsz_outer(im, jm, km, hw));
}

// halo_exchange.cl:156-291 (inner=0) / halo_exchange_correct.cl read (inner=1)
void oracle_halo_pack(const float *a, float *buf, unsigned im, unsigned jm, unsigned km,
                      unsigned hw, unsigned vdim, size_t es, size_t vs, int inner) {
    const unsigned top = (im > jm ? im : jm);
    const size_t v_sz = inner ? vsz_inner(im, jm, km, hw) : vsz_outer(im, jm, km, hw);
    for (unsigned gl = 0; gl < km * top; ++gl) {
        const unsigned k = gl % km, i = gl / km;
        for (unsigned v = 0; v < vdim; ++v)
            for (unsigned w = 0; w < hw; ++w) {
                auto A = [&](size_t idx) { return a[idx * es + v * vs]; };
                if (!inner) {
                    if (i < im && k < km) {
                        buf[v * v_sz + i + (size_t)im * w + (size_t)k * im * hw] =
                            A(i + (size_t)im * w + (size_t)k * im * jm);
                        buf[v * v_sz + (size_t)km * im * hw + i + (size_t)im * w + (size_t)k * im * hw] =
                            A(i + (size_t)im * w + (size_t)k * im * jm + (size_t)im * (jm - hw));
                    }
                    if (i < jm - hw && k < km && i > hw - 1) {
                        buf[v * v_sz + (size_t)km * im * hw * 2 + (size_t)(i - hw) * hw + w +
                            (size_t)k * (jm - 2 * hw) * hw] = A((size_t)i * im + w + (size_t)k * im * jm);
                        buf[v * v_sz + (size_t)km * im * hw * 2 + (size_t)km * (jm - 2 * hw) * hw +
                            (size_t)(i - hw) * hw + w + (size_t)k * (jm - 2 * hw) * hw] =
                            A((size_t)i * im + w + (size_t)k * im * jm + im - hw);
                    }
                } else {
                    const size_t ni = im - 2 * hw;
                    if (i < im - hw && k < km && i > hw - 1) {
                        buf[v * v_sz + (i - hw) + ni * w + (size_t)k * ni * hw] =
                            A((size_t)im * hw + i + (size_t)im * w + (size_t)k * im * jm);
                        buf[v * v_sz + (size_t)km * ni * hw + (i - hw) + ni * w + (size_t)k * ni * hw] =
                            A(i + (size_t)k * im * jm + (size_t)im * (jm - 2 * hw) + (size_t)im * w);
                    }
                    if (i < jm - hw && k < km && i > hw - 1) {
                        buf[v * v_sz + (size_t)km * ni * hw * 2 + (size_t)(i - hw) * hw + w +
                            (size_t)k * (jm - 2 * hw) * hw] =
                            A((size_t)i * im + w + hw + (size_t)k * im * jm);
                        buf[v * v_sz + (size_t)km * ni * hw * 2 + (size_t)km * (jm - 2 * hw) * hw +
                            (size_t)(i - hw) * hw + w + (size_t)k * (jm - 2 * hw) * hw] =
                            A((size_t)i * im + w + (size_t)k * im * jm + im - 2 * hw);
                    }
                }
            }
    }
}

// halo_exchange.cl:3-152 (inner=0) / halo_exchange_correct.cl write (inner=1)
void oracle_halo_unpack(float *a, const float *buf, unsigned im, unsigned jm, unsigned km,
                        unsigned hw, unsigned vdim, size_t es, size_t vs, int inner) {
    const unsigned top = (im > jm ? im : jm);
    const size_t v_sz = vsz_outer(im, jm, km, hw);
    for (unsigned gl = 0; gl < km * top; ++gl) {
        const unsigned k = gl % km, i = gl / km;
        for (unsigned v = 0; v < vdim; ++v)
            for (unsigned w = 0; w < hw; ++w) {
                auto A = [&](size_t idx) -> float & { return a[idx * es + v * vs]; };
                const size_t wrow = inner ? 0 : (size_t)im * w;
                if (i < im && k < km) {
                    A(i + (size_t)im * w + (size_t)k * im * jm) =
                        buf[v * v_sz + i + wrow + (size_t)k * im * hw];
                    A(i + (size_t)im * w + (size_t)k * im * jm + (size_t)im * (jm - hw)) =
                        buf[v * v_sz + (size_t)km * im * hw + i + wrow + (size_t)k * im * hw];
                }
                if (i < jm - hw && k < km && i > hw - 1) {
                    A((size_t)i * im + w + (size_t)k * im * jm) =
                        buf[v * v_sz + (size_t)km * im * hw * 2 + (size_t)(i - hw) * hw + w +
                            (size_t)k * (jm - 2 * hw) * hw];
                    A((size_t)i * im + w + (size_t)k * im * jm + im - hw) =
                        buf[v * v_sz + (size_t)km * im * hw * 2 + (size_t)km * (jm - 2 * hw) * hw +
                            (size_t)(i - hw) * hw + w + (size_t)k * (jm - 2 * hw) * hw];
                }
            }
    }
}

}  // extern "C"
