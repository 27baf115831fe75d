// solnio.cu -- E-field solution files in the reference's binary layout.
//
// write_solnVectorMTX / read_solnVectorMTX (f90/3D_MT/ioMod/ioAscii.f90:
// 493-597) with FileWriteInit / FileReadInit (:188-215;
// f90/3D_MT/ioMod/ioBinary.f90:61-93) and EfileWrite / EfileRead
// (ioBinary.f90:314-368).  The file is a Fortran unformatted sequential file
// as gfortran writes it: every record is framed by its length in bytes as a
// little-endian int32 before and after.  Records:
//   1  version (20 chars), nTx, nMode, nx, ny, nz, nzAir (int32),
//      ox, oy, oz, rotdeg (float64)
//   2  dx[nx]   3  dy[ny]   4  dz[nz] (air layers first)
// then, for each transmitter j = 1..nTx and polarisation k = 1..nMode,
//   omega (float64), j, k (int32), polarisation name (20 chars)
//   Ex [nx][ny+1][nz+1], Ey, Ez (complex128, x fastest)
// so the record of (j, k) follows 4 + ((j-1) nMode + (k-1)) 4 records
// (EfileRead's nRecSkip).  The three field records are the three blocks of a
// full edge vector.  Records longer than 2^31 - 1 bytes would need
// gfortran's sub-records and are refused.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "solver.h"

namespace mt3d {

namespace {

constexpr int64_t kMaxRecord = 2147483647LL;

struct File {
    FILE *f = nullptr;
    ~File()
    {
        if (f) fclose(f);
    }
};

bool put_record(FILE *f, const void *p, int64_t n)
{
    const int32_t m = (int32_t)n;
    return fwrite(&m, 4, 1, f) == 1 && (n == 0 || fwrite(p, 1, (size_t)n, f) == (size_t)n) && fwrite(&m, 4, 1, f) == 1;
}

// reads the next record into p (n bytes expected); n < 0: skip whatever it holds
bool get_record(FILE *f, void *p, int64_t n, int64_t *got = nullptr)
{
    int32_t a = 0, b = 0;
    if (fread(&a, 4, 1, f) != 1 || a < 0) return false;
    if (got) *got = a;
    if (n < 0) {
        if (fseek(f, a, SEEK_CUR) != 0) return false;
    } else {
        if (a != n) return false;
        if (n > 0 && fread(p, 1, (size_t)n, f) != (size_t)n) return false;
    }
    return fread(&b, 4, 1, f) == 1 && a == b;
}

void pad20(char *dst, const char *src)
{
    memset(dst, ' ', 20);
    if (src) memcpy(dst, src, std::min<size_t>(20, strlen(src)));
}

#pragma pack(push, 1)
struct Header {
    char version[20];
    int32_t nTx, nMode, nx, ny, nz, nzAir;
    double ox, oy, oz, rotdeg;
};
struct TxHeader {
    double omega;
    int32_t iTx, iMode;
    char name[20];
};
#pragma pack(pop)
static_assert(sizeof(Header) == 76, "header record");
static_assert(sizeof(TxHeader) == 36, "transmitter record");

}  // namespace

int read_soln_header(const char *path, int *nTx, int *nMode, int *nx, int *ny, int *nz, int *nzAir, double *origin,
                     double *rotdeg, double *dx, double *dy, double *dz, std::string &err)
{
    File fl;
    if (!path || !(fl.f = fopen(path, "rb"))) {
        err = std::string("cannot open ") + (path ? path : "(null)");
        return 5;
    }
    Header h;
    if (!get_record(fl.f, &h, sizeof h) || h.nx < 1 || h.ny < 1 || h.nz < 1 || h.nTx < 0 || h.nMode < 0) {
        err = "not a solution file (header record)";
        return 5;
    }
    if (nTx) *nTx = h.nTx;
    if (nMode) *nMode = h.nMode;
    if (nx) *nx = h.nx;
    if (ny) *ny = h.ny;
    if (nz) *nz = h.nz;
    if (nzAir) *nzAir = h.nzAir;
    if (origin) {
        origin[0] = h.ox;
        origin[1] = h.oy;
        origin[2] = h.oz;
    }
    if (rotdeg) *rotdeg = h.rotdeg;
    std::vector<double> tmp;
    double *out[3] = {dx, dy, dz};
    const int n[3] = {h.nx, h.ny, h.nz};
    for (int a = 0; a < 3; a++) {
        tmp.resize(n[a]);
        if (!get_record(fl.f, tmp.data(), (int64_t)n[a] * 8)) {
            err = "not a solution file (grid records)";
            return 5;
        }
        if (out[a]) memcpy(out[a], tmp.data(), (size_t)n[a] * 8);
    }
    return 0;
}

int Solver::write_soln(const char *path, int nTx, int nPol, const double *omegas, const double *origin, double rotdeg,
                       const double *e, bool device)
{
    if (!path || nTx < 1 || nPol < 1 || !omegas || !e) return fail(5, "mt3d_write_soln: invalid arguments");
    const int64_t nX = (int64_t)nx * (ny + 1) * (nz + 1), nY = (int64_t)(nx + 1) * ny * (nz + 1),
                  nZ = (int64_t)(nx + 1) * (ny + 1) * nz;
    if (std::max(nX, std::max(nY, nZ)) * 16 > kMaxRecord)
        return fail(5, "mt3d_write_soln: a field component exceeds the 2 GiB record limit");
    File fl;
    if (!(fl.f = fopen(path, "wb"))) return fail(5, std::string("mt3d_write_soln: cannot create ") + path);
    Header h;
    pad20(h.version, "");
    h.nTx = nTx;
    h.nMode = nPol;
    h.nx = nx;
    h.ny = ny;
    h.nz = nz;
    h.nzAir = nzAir;
    h.ox = origin ? origin[0] : 0.0;
    h.oy = origin ? origin[1] : 0.0;
    h.oz = origin ? origin[2] : 0.0;
    h.rotdeg = rotdeg;
    bool ok = put_record(fl.f, &h, sizeof h) && put_record(fl.f, dx_.data(), (int64_t)nx * 8) &&
              put_record(fl.f, dy_.data(), (int64_t)ny * 8) && put_record(fl.f, dz_.data(), (int64_t)nz * 8);
    // create_solnVector names the two MT polarisations Ex and Ey
    static const char *names[2] = {"Ex", "Ey"};
    std::vector<double2> stage;
    if (device) stage.resize((size_t)nE);
    for (int j = 0; ok && j < nTx; j++)
        for (int k = 0; ok && k < nPol; k++) {
            TxHeader t;
            t.omega = omegas[j];
            t.iTx = j + 1;
            t.iMode = k + 1;
            pad20(t.name, nPol == 2 ? names[k] : "");
            const double2 *src = reinterpret_cast<const double2 *>(e) + ((size_t)j * nPol + k) * nE;
            if (device) {
                if (int rc = check(cudaMemcpy(stage.data(), src, nE * sizeof(double2), cudaMemcpyDeviceToHost),
                                   "mt3d_write_soln"))
                    return rc;
                src = stage.data();
            }
            ok = put_record(fl.f, &t, sizeof t) && put_record(fl.f, src, nX * 16) &&
                 put_record(fl.f, src + nX, nY * 16) && put_record(fl.f, src + nX + nY, nZ * 16);
        }
    if (!ok || fflush(fl.f) != 0) return fail(5, std::string("mt3d_write_soln: write failed on ") + path);
    return 0;
}

int Solver::read_soln(const char *path, int iTx, int iPol, double *omega, double *e, bool device)
{
    if (!path || iTx < 1 || iPol < 1 || !e) return fail(5, "mt3d_read_soln: invalid arguments");
    File fl;
    if (!(fl.f = fopen(path, "rb"))) return fail(5, std::string("mt3d_read_soln: cannot open ") + path);
    Header h;
    if (!get_record(fl.f, &h, sizeof h)) return fail(5, "mt3d_read_soln: not a solution file (header record)");
    // CheckgridConsist (ioBinary.f90:95-130): grid sizes must agree
    if (h.nx != nx || h.ny != ny || h.nz != nz || h.nzAir != nzAir)
        return fail(5, "mt3d_read_soln: grid size of the file differs from the handle's");
    if (iTx > h.nTx || iPol > h.nMode) return fail(5, "mt3d_read_soln: transmitter or polarisation not in the file");
    const int64_t nX = (int64_t)nx * (ny + 1) * (nz + 1), nY = (int64_t)(nx + 1) * ny * (nz + 1),
                  nZ = (int64_t)(nx + 1) * (ny + 1) * nz;
    const int64_t skip = (int64_t)((iTx - 1) * h.nMode + (iPol - 1)) * 4 + 3;  // grid records + earlier fields
    for (int64_t r = 0; r < skip; r++)
        if (!get_record(fl.f, nullptr, -1)) return fail(5, "mt3d_read_soln: file ends early");
    TxHeader t;
    if (!get_record(fl.f, &t, sizeof t) || t.iTx != iTx || t.iMode != iPol)
        return fail(5, "mt3d_read_soln: transmitter record not found");
    std::vector<double2> stage;
    double2 *dst = reinterpret_cast<double2 *>(e);
    if (device) {
        stage.resize((size_t)nE);
        dst = stage.data();
    }
    if (!get_record(fl.f, dst, nX * 16) || !get_record(fl.f, dst + nX, nY * 16) ||
        !get_record(fl.f, dst + nX + nY, nZ * 16))
        return fail(5, "mt3d_read_soln: field records do not match the grid");
    if (device)
        if (int rc = check(cudaMemcpy(e, stage.data(), nE * sizeof(double2), cudaMemcpyHostToDevice), "mt3d_read_soln"))
            return rc;
    if (omega) *omega = t.omega;
    return 0;
}

}  // namespace mt3d
