// Checkpoint files in the reference's formats (host I/O, native byte order,
// FP64, fields x fastest):
//   SolutionDump.<step>  (CurvilinearCSolver::dumpSolution,
//                         src/CurvilinearCSolver_Core.cpp:1333-1405): 5 header
//                         values (time step, time, Nx, Ny, Nz), then x, y, z,
//                         rho, rhoU, rhoV, rhoW, rhoE;
//   SpongeAvgDump.<step> (SpongeBC::dumpSpongeAvg, src/SpongeBC.cpp:363-424):
//                         the five sponge target fields, no header.
#include <cstdio>
#include <string>

#include "mc3d_internal.h"

namespace mc3d {

namespace {
struct File {
    FILE *f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};
}  // namespace

int write_solution_dump(const char *path, int time_step, double time, int Nx, int Ny, int Nz,
                        const double *const fields[8]) {
    const size_t n = (size_t)Nx * Ny * Nz;
    File fl;
    if (!(fl.f = fopen(path, "wb"))) return fail(MC3D_ERR_ARG, std::string("cannot write ") + path);
    const double hdr[5] = {(double)time_step, time, (double)Nx, (double)Ny, (double)Nz};
    if (fwrite(hdr, sizeof(double), 5, fl.f) != 5) return fail(MC3D_ERR_ARG, std::string("write failed: ") + path);
    for (int k = 0; k < 8; k++)
        if (fwrite(fields[k], sizeof(double), n, fl.f) != n)
            return fail(MC3D_ERR_ARG, std::string("write failed: ") + path);
    return MC3D_OK;
}

int read_solution_header(const char *path, int *time_step, double *time, int *Nx, int *Ny, int *Nz) {
    File fl;
    if (!(fl.f = fopen(path, "rb"))) return fail(MC3D_ERR_ARG, std::string("Couldn't open file ") + path);
    double h[5];
    if (fread(h, sizeof(double), 5, fl.f) != 5) return fail(MC3D_ERR_ARG, std::string("short header: ") + path);
    // src/MPI_3DCompact.cpp:97-101 casts the header values to int
    if (time_step) *time_step = (int)h[0];
    if (time) *time = h[1];
    if (Nx) *Nx = (int)h[2];
    if (Ny) *Ny = (int)h[3];
    if (Nz) *Nz = (int)h[4];
    return MC3D_OK;
}

int read_solution_fields(const char *path, long long n, double *const fields[8]) {
    int Nx, Ny, Nz;
    int rc = read_solution_header(path, nullptr, nullptr, &Nx, &Ny, &Nz);
    if (rc) return rc;
    if ((long long)Nx * Ny * Nz != n) return fail(MC3D_ERR_CONFIG, std::string("grid size differs from ") + path);
    File fl;
    if (!(fl.f = fopen(path, "rb"))) return fail(MC3D_ERR_ARG, std::string("Couldn't open file ") + path);
    for (int k = 0; k < 8; k++) {
        const long long off = (5 + (long long)k * n) * (long long)sizeof(double);
        if (!fields[k]) continue;
        if (fseek(fl.f, (long)off, SEEK_SET) != 0 || fread(fields[k], sizeof(double), (size_t)n, fl.f) != (size_t)n)
            return fail(MC3D_ERR_ARG, std::string("short file: ") + path);
    }
    return MC3D_OK;
}

int write_sponge_avg(const char *path, long long n, const double *const fields[5]) {
    File fl;
    if (!(fl.f = fopen(path, "wb"))) return fail(MC3D_ERR_ARG, std::string("cannot write ") + path);
    for (int k = 0; k < 5; k++)
        if (fwrite(fields[k], sizeof(double), (size_t)n, fl.f) != (size_t)n)
            return fail(MC3D_ERR_ARG, std::string("write failed: ") + path);
    return MC3D_OK;
}

int read_sponge_avg(const char *path, long long n, double *const fields[5]) {
    File fl;
    if (!(fl.f = fopen(path, "rb"))) return fail(MC3D_ERR_ARG, std::string("Couldn't open file ") + path);
    for (int k = 0; k < 5; k++)
        if (fread(fields[k], sizeof(double), (size_t)n, fl.f) != (size_t)n)
            return fail(MC3D_ERR_ARG, std::string("short file: ") + path);
    return MC3D_OK;
}

}  // namespace mc3d

extern "C" {

int mc3d_dump_read_header(const char *path, int *time_step, double *time, int *Nx, int *Ny, int *Nz) {
    if (!path) return mc3d::fail(MC3D_ERR_ARG, "null path");
    return mc3d::read_solution_header(path, time_step, time, Nx, Ny, Nz);
}

int mc3d_dump_read_fields(const char *path, long long n, double *const fields[8]) {
    if (!path || !fields || n <= 0) return mc3d::fail(MC3D_ERR_ARG, "bad argument");
    return mc3d::read_solution_fields(path, n, fields);
}

int mc3d_dump_write(const char *path, int time_step, double time, int Nx, int Ny, int Nz,
                    const double *const fields[8]) {
    if (!path || !fields || Nx <= 0 || Ny <= 0 || Nz <= 0) return mc3d::fail(MC3D_ERR_ARG, "bad argument");
    for (int k = 0; k < 8; k++)
        if (!fields[k]) return mc3d::fail(MC3D_ERR_ARG, "null field");
    return mc3d::write_solution_dump(path, time_step, time, Nx, Ny, Nz, fields);
}

}  // extern "C"
