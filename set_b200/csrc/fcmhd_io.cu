// fcmhd_io.cu -- the reference's on-disk formats (host code).
//
// Grid/state stream file: written by SET_Gelios/source/Setka.cpp:1158-1567, read by the FCMHD
// host in Set_Storage (SET_Fortran_Cuda_MHD/Storage_module.f90:42-100).  Unformatted stream, no
// record markers, native byte order, in this order:
//   real(8) time_all; integer(4) N_cell; integer(4) N_gran;
//   real(8) Cell_par(16,N); real(8) Cell_center(3,N); real(8) Cell_Volume(N);
//   integer(4) Cell_gran(6,N);
//   real(8) Gran_normal(3,G); real(8) Gran_square(G); real(8) Gran_center(3,G);
//   integer(4) Gran_neighbour(2,G); integer(4) Gran_neighbour_TVD(2,G);
//   real(8) 121.0; integer(4) Gran_type(G); real(8) 122.0; real(8) Gran_POTOK(9,G); real(8) 123.0
// Checkpoint: Save_Storage / Fill_data (Storage_module.f90:160-209):
//   real(8) time_all; real(8) Cell_par(16,N); real(8) 321.0
// Every read checks the sentinels and the file length; a mismatch is SETB_EIO.
#include <cstdio>
#include <cstring>
#include <vector>

#include "setb200.h"

namespace {

struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(path ? std::fopen(path, mode) : nullptr) {}
    ~File() {
        if (f) std::fclose(f);
    }
    bool read(void* p, size_t bytes) { return bytes == 0 || std::fread(p, 1, bytes, f) == bytes; }
    bool write(const void* p, size_t bytes) { return bytes == 0 || std::fwrite(p, 1, bytes, f) == bytes; }
    bool sentinel(double want) {
        double v = 0.0;
        return read(&v, sizeof v) && v == want;
    }
    bool at_end() { return std::fgetc(f) == EOF; }
};

bool write_d(File& f, double v) { return f.write(&v, sizeof v); }

}  // namespace

extern "C" {

int32_t setb_fcmhd_read_header(const char* path, double* time_all, int32_t* n_cell, int32_t* n_gran) {
    if (!path || !time_all || !n_cell || !n_gran) return SETB_EINVAL;
    File f(path, "rb");
    if (!f.f) return SETB_EIO;
    if (!f.read(time_all, 8) || !f.read(n_cell, 4) || !f.read(n_gran, 4)) return SETB_EIO;
    if (*n_cell < 1 || *n_gran < 1) return SETB_EIO;
    return SETB_OK;
}

int32_t setb_fcmhd_read(const char* path, int32_t n_cell, int32_t n_gran, double* time_all, double* cell_par,
                        double* cell_center, double* cell_volume,
                        int32_t* cell_gran, double* gran_normal, double* gran_square, double* gran_center,
                        int32_t* gran_neighbour, int32_t* gran_neighbour_tvd, int32_t* gran_type, double* gran_potok) {
    if (!path || !time_all || !cell_par || !cell_center || !cell_volume || !cell_gran || !gran_normal || !gran_square ||
        !gran_center || !gran_neighbour || !gran_neighbour_tvd || !gran_type)
        return SETB_EINVAL;
    File f(path, "rb");
    if (!f.f) return SETB_EIO;
    int32_t N = 0, G = 0;
    if (!f.read(time_all, 8) || !f.read(&N, 4) || !f.read(&G, 4) || N < 1 || G < 1) return SETB_EIO;
    if (N != n_cell || G != n_gran) return SETB_EIO;   // the caller's buffers hold n_cell / n_gran
    const size_t n = (size_t)N, g = (size_t)G;
    bool ok = f.read(cell_par, 8 * 16 * n) && f.read(cell_center, 8 * 3 * n) && f.read(cell_volume, 8 * n) &&
              f.read(cell_gran, 4 * 6 * n) && f.read(gran_normal, 8 * 3 * g) && f.read(gran_square, 8 * g) &&
              f.read(gran_center, 8 * 3 * g) && f.read(gran_neighbour, 4 * 2 * g) &&
              f.read(gran_neighbour_tvd, 4 * 2 * g) && f.sentinel(121.0) && f.read(gran_type, 4 * g) &&
              f.sentinel(122.0);
    if (!ok) return SETB_EIO;
    if (gran_potok) {
        if (!f.read(gran_potok, 8 * 9 * g)) return SETB_EIO;
    } else {
        std::vector<double> skip(9 * g);
        if (!f.read(skip.data(), 8 * 9 * g)) return SETB_EIO;
    }
    if (!f.sentinel(123.0) || !f.at_end()) return SETB_EIO;
    return SETB_OK;
}

int32_t setb_fcmhd_write(const char* path, double time_all, int32_t n_cell, int32_t n_gran, const double* cell_par,
                         const double* cell_center, const double* cell_volume, const int32_t* cell_gran,
                         const double* gran_normal, const double* gran_square, const double* gran_center,
                         const int32_t* gran_neighbour, const int32_t* gran_neighbour_tvd, const int32_t* gran_type,
                         const double* gran_potok) {
    if (!path || n_cell < 1 || n_gran < 1 || !cell_par || !cell_center || !cell_volume || !cell_gran || !gran_normal ||
        !gran_square || !gran_center || !gran_neighbour || !gran_neighbour_tvd || !gran_type)
        return SETB_EINVAL;
    File f(path, "wb");
    if (!f.f) return SETB_EIO;
    const size_t n = (size_t)n_cell, g = (size_t)n_gran;
    std::vector<double> zeros(gran_potok ? 0 : 9 * g, 0.0);   // Setka.cpp writes zero fluxes
    bool ok = write_d(f, time_all) && f.write(&n_cell, 4) && f.write(&n_gran, 4) && f.write(cell_par, 8 * 16 * n) &&
              f.write(cell_center, 8 * 3 * n) && f.write(cell_volume, 8 * n) && f.write(cell_gran, 4 * 6 * n) &&
              f.write(gran_normal, 8 * 3 * g) && f.write(gran_square, 8 * g) && f.write(gran_center, 8 * 3 * g) &&
              f.write(gran_neighbour, 4 * 2 * g) && f.write(gran_neighbour_tvd, 4 * 2 * g) && write_d(f, 121.0) &&
              f.write(gran_type, 4 * g) && write_d(f, 122.0) &&
              f.write(gran_potok ? gran_potok : zeros.data(), 8 * 9 * g) && write_d(f, 123.0);
    return ok ? SETB_OK : SETB_EIO;
}

int32_t setb_checkpoint_write(const char* path, double time_all, int32_t n_cell, const double* cell_par) {
    if (!path || n_cell < 1 || !cell_par) return SETB_EINVAL;
    File f(path, "wb");
    if (!f.f) return SETB_EIO;
    const bool ok = write_d(f, time_all) && f.write(cell_par, 8 * 16 * (size_t)n_cell) && write_d(f, 321.0);
    return ok ? SETB_OK : SETB_EIO;
}

int32_t setb_checkpoint_read(const char* path, int32_t n_cell, double* time_all, double* cell_par) {
    if (!path || n_cell < 1 || !time_all || !cell_par) return SETB_EINVAL;
    File f(path, "rb");
    if (!f.f) return SETB_EIO;
    const bool ok = f.read(time_all, 8) && f.read(cell_par, 8 * 16 * (size_t)n_cell) && f.sentinel(321.0) && f.at_end();
    return ok ? SETB_OK : SETB_EIO;
}

}  // extern "C"
