// ssf_manager.hpp -- TEST INFRASTRUCTURE ONLY. Placed ahead of the reference's
// include/ on the include path when src/MC.cpp is compiled into oracle/_ref/,
// so that MC.cpp's #include "ssf_manager.hpp" finds this file instead of the
// real manager (which needs lattice_lib's FFTW-backed Fourier module).
// MC.cpp uses only the per-component transforms FT_S{x,y,z}_t in
// save_ft_spin_state, which the compiled reference is never asked to run:
// these stand-ins hold empty buffers and transform nothing.
#pragma once
#include <complex>
#include <vector>

#include "MC.hpp"

template <typename T>
struct FourierBuffer {
    int num_sublattices = 0;
    ivec3_t k_dims{0, 0, 0};
    std::vector<std::vector<std::complex<double>>> data;
    const std::vector<std::complex<double>>& operator[](size_t sl) const { return data[sl]; }
};

struct FT_S_stub {
    FourierBuffer<CMC::HeisenbergSpin> buf;
    explicit FT_S_stub(CMC::Lattice&) {}
    void transform() {}
    const FourierBuffer<CMC::HeisenbergSpin>& get_buffer() const { return buf; }
};
struct FT_Sx_t : FT_S_stub {
    using FT_S_stub::FT_S_stub;
};
struct FT_Sy_t : FT_S_stub {
    using FT_S_stub::FT_S_stub;
};
struct FT_Sz_t : FT_S_stub {
    using FT_S_stub::FT_S_stub;
};
