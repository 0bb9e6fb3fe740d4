// tmx_writers.cpp -- the reference's Tecplot text files, written from the
// state after the last step (tmx_write_file in include/tmx.h).  Host code
// over the public C ABI: the fields come from tmx_fields, the numbers from
// tmx_pressure_power and tmx_mixing; the lines are printed with the
// reference's own formats so that the files match the reference's byte for
// byte when the fields do (the plain FP64 form).
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/tmx.h"

namespace tmx_host {
int fail(int code, const char* fmt, ...);
}
using tmx_host::fail;

namespace {

// The seven fields of both boxes in the reference's [i][j][k] order.
struct Fields {
    int inx, iny, nz, mnx, mny, ia, ib;
    std::vector<double> f[2][7];
    double at(int b, int fld, int i, int j, int k) const
    {
        const int ny = b ? mny : iny;
        return f[b][fld][((size_t)(i - 1) * ny + (j - 1)) * nz + (k - 1)];
    }
};

int load_fields(tmx_handle* h, const tmx_case& c, Fields& F)
{
    F.inx = c.inx;
    F.iny = c.iny;
    F.nz = c.nz;
    F.mnx = c.mnx;
    F.mny = c.mny;
    F.ia = c.ia;
    F.ib = c.ia + c.mnx - 1;
    for (int b = 0; b < 2; b++) {
        const size_t n = (size_t)(b ? c.mnx : c.inx) * (b ? c.mny : c.iny) * c.nz;
        for (int fld = 0; fld < 7; fld++) {
            F.f[b][fld].resize(n);
            int rc = tmx_fields(h, b, fld, F.f[b][fld].data());
            if (rc) return rc;
        }
    }
    return TMX_OK;
}

// field ids in the order the files list them
constexpr int RHO = TMX_RHO, UX = TMX_UX, UY = TMX_UY, UZ = TMX_UZ, CA = TMX_CA, CB = TMX_CB, CC = TMX_CC;

// write_Domain_Data (Tmixer.cpp:10028-10064); the mixing zone's header
// repeats the inlet box's sizes, as the reference's does.
void domain_data(FILE* fp, const Fields& F)
{
    std::fprintf(fp, "VARIABLES = X\tY\tZ\tUx\tUy\tUz\trho\tgrho\thrho\tprho\r\n");
    std::fprintf(fp, "ZONE T= \"Horizontal Channel\"  I=%d,J=%d,K=%d  \r\n", F.inx, F.iny, F.nz);
    for (int i = 1; i <= F.inx; i++) {
        for (int j = 1; j <= F.iny; j++) {
            for (int k = 1; k <= F.nz; k++)
                std::fprintf(fp, "%d\t%d\t%d\t%lf\t%lf\t%lf\t%lf\t%lf\t%lf\t%lf\n", i, j + F.mny, k, F.at(0, UX, i, j, k),
                             F.at(0, UY, i, j, k), F.at(0, UZ, i, j, k), F.at(0, RHO, i, j, k), F.at(0, CA, i, j, k),
                             F.at(0, CB, i, j, k), F.at(0, CC, i, j, k));
            std::fprintf(fp, "\n");
        }
        std::fprintf(fp, "\n");
    }
    std::fprintf(fp, "ZONE T= \"Mixing Channel \" I=%d,J=%d,K=%d  \r\n", F.inx, F.iny, F.nz);
    for (int i = 1; i <= F.mnx; i++) {
        for (int j = 1; j <= F.mny; j++) {
            for (int k = 1; k <= F.nz; k++)
                std::fprintf(fp, "%d\t%d\t%d\t%lf\t%lf\t%lf\t%lf\t%lf\t%lf\t%lf\n", i, j, k, F.at(1, UX, i, j, k),
                             F.at(1, UY, i, j, k), F.at(1, UZ, i, j, k), F.at(1, RHO, i, j, k), F.at(1, CA, i, j, k),
                             F.at(1, CB, i, j, k), F.at(1, CC, i, j, k));
            std::fprintf(fp, "\n");
        }
        std::fprintf(fp, "\n");
    }
}

void pvc_line(FILE* fp, int a, int b, double u, double v, const Fields& F, int box, int i, int j, int k)
{
    std::fprintf(fp, "%d\t%d\t%lf\t%lf\t%lf\t%lf\t%lf\t%lf\n", a, b, u, v, F.at(box, RHO, i, j, k), F.at(box, CA, i, j, k),
                 F.at(box, CB, i, j, k), F.at(box, CC, i, j, k));
}

// write_Data_P_V_C (Tmixer.cpp:10065-10160).  Three of its sections read
// fixed rows (mixing row 600, mixing row mny-1 and inlet row 775-mny); a
// section whose row lies outside its box (the reference would read outside
// its arrays there) is left out.
void data_pvc(FILE* fp, const Fields& F)
{
    std::fprintf(fp, "VARIABLES = 'X','Y','Ux','Uy','rho','Ca','Cb','Cc'\r\n");
    std::fprintf(fp, "ZONE T=\"Inlet Channel\" \r\n");
    int zc = (F.nz + 1) / 2;
    for (int i = 1; i <= F.inx; i++) {
        for (int j = F.mny + 1; j <= F.iny + F.mny; j++)
            pvc_line(fp, i, j, F.at(0, UX, i, j - F.mny, zc), F.at(0, UY, i, j - F.mny, zc), F, 0, i, j - F.mny, zc);
        std::fprintf(fp, "\n");
    }
    std::fprintf(fp, "ZONE T=\"Mixing Channel\"\r\n");
    for (int i = F.ia; i <= F.ib; i++) {
        for (int j = 1; j <= F.mny + 1; j++) {
            if (j == F.mny + 1)
                pvc_line(fp, i, j, F.at(0, UX, i, j - F.mny, zc), F.at(0, UY, i, j - F.mny, zc), F, 0, i, j - F.mny, zc);
            else
                pvc_line(fp, i, j, F.at(1, UX, i - F.ia + 1, j, zc), F.at(1, UY, i - F.ia + 1, j, zc), F, 1,
                         i - F.ia + 1, j, zc);
        }
        std::fprintf(fp, "\n");
    }
    std::fprintf(fp, "ZONE T=\"InletCrossSectionY_Z(Z_%d,Y_%d)\"\r\n", F.nz, F.iny);
    for (int j = 1; j <= F.iny; j++) {
        for (int k = 1; k <= F.nz; k++) pvc_line(fp, j, k, F.at(0, UX, 1, j, k), F.at(0, UZ, 1, j, k), F, 0, 1, j, k);
        std::fprintf(fp, "\n");
    }
    zc = 2;  // outlet
    std::fprintf(fp, "ZONE T=\"Outlet_Z_X%d(Z_%d,X_%d)\"\r\n", zc, F.nz, F.mnx);
    for (int i = 1; i <= F.nz; i++) {
        for (int j = 1; j <= F.mnx; j++) pvc_line(fp, i, j, F.at(1, UX, j, zc, i), F.at(1, UZ, j, zc, i), F, 1, j, zc, i);
        std::fprintf(fp, "\n");
    }
    const int rows[2] = {600, F.mny - 1};
    for (int r = 0; r < 2; r++) {
        zc = rows[r];
        if (zc < 1 || zc > F.mny) continue;
        std::fprintf(fp, "ZONE T=\"MixingZ_X_%d(Z_%d,X_%d)\"\r\n", zc, F.nz, F.mnx);
        for (int i = 1; i <= F.nz; i++) {
            for (int j = 1; j <= F.mnx; j++)
                pvc_line(fp, i, j, F.at(1, UZ, j, zc, i), F.at(1, UX, j, zc, i), F, 1, j, zc, i);
            std::fprintf(fp, "\n");
        }
    }
    zc = 775 - F.mny;
    if (zc >= 1 && zc <= F.iny) {
        std::fprintf(fp, "ZONE T=\"MixingZ_X_%d(Z_%d,X_%d)\"\r\n", zc + F.mny, F.nz, F.mnx);
        for (int k = 1; k <= F.nz; k++) {
            for (int i = 1; i <= F.inx; i++)
                pvc_line(fp, k, i, F.at(0, UZ, i, zc, k), F.at(0, UX, i, zc, k), F, 0, i, zc, k);
            std::fprintf(fp, "\n");
        }
    }
}

// the Pressure file of write_Pressure_Power (Tmixer.cpp:9866-10027)
int pressure_file(FILE* fp, tmx_handle* h, const tmx_case& c)
{
    std::vector<double> prow((size_t)(c.mny + c.iny) * 3), px((size_t)c.inx * 2), pw((size_t)(c.mny - 2) * 5);
    double u[2];
    int rc = tmx_pressure_power(h, prow.data(), px.data(), pw.data(), u);
    if (rc) return rc;
    std::fprintf(fp, "ZONE T=\"PressureAlongMixingChannel\" \r\n");
    for (int r = 0; r < c.mny + c.iny; r++) {
        const double t = prow[3 * r + 1], d = prow[3 * r + 2];
        std::fprintf(fp, "%d\t%g\t%g\t%g\n", (int)prow[3 * r], t, t * u[0], d * u[0]);
    }
    std::fprintf(fp, "ZONE T=\"HorizontalSectionPressure\" \r\n");
    for (int i = 0; i < c.inx; i++)
        std::fprintf(fp, "%d\t%g\t%g\t%g\n", (int)px[2 * i], px[2 * i + 1], px[2 * i + 1] * u[0], 0.0);
    std::fprintf(fp, "ZONE T=\"SpecificPower\"\n");
    for (int j = 0; j < c.mny - 2; j++)
        std::fprintf(fp, "%d\t%g\t%g\t%g\n", (int)pw[5 * j], pw[5 * j + 1], pw[5 * j + 1] * u[1], pw[5 * j + 2] * u[1]);
    return TMX_OK;
}

// the MixingQuality file of write_MixingQuality (Tmixer.cpp:10161-10409)
int mixing_file(FILE* fp, tmx_handle* h, const tmx_case& c)
{
    std::vector<double> rows((size_t)(c.mny + c.iny) * 7);
    int rc = tmx_mixing(h, rows.data(), nullptr);
    if (rc) return rc;
    std::fprintf(fp, "ZONE T=\"Mixing Quality\" \r\n");
    std::fprintf(fp, "VARIABLES= \"Y\"\"A\"\"B\"\"C\"\"IA\"\"IB\"\"IC\"\r\n");
    for (int r = 0; r < c.mny + c.iny; r++) {
        const double* o = &rows[7 * (size_t)r];
        std::fprintf(fp, "%d\t%g\t%g\t%g\t%g\t%g\t%g\n", (int)o[0], o[1], o[2], o[3], o[4], o[5], o[6]);
    }
    return TMX_OK;
}

}  // namespace

extern "C" int tmx_write_file(tmx_handle* h, int kind, const char* path)
{
    if (!h || !path) return fail(TMX_E_INVALID, "null argument");
    if (kind < TMX_FILE_DOMAIN || kind > TMX_FILE_MIXING) return fail(TMX_E_INVALID, "unknown file kind %d", kind);
    tmx_case cs;
    int rc0 = tmx_case_of(h, &cs);
    if (rc0) return rc0;
    const tmx_case* c = &cs;
    FILE* fp = std::fopen(path, "w");
    if (!fp) return fail(TMX_E_INVALID, "cannot open %s for writing", path);
    int rc = TMX_OK;
    if (kind == TMX_FILE_DOMAIN || kind == TMX_FILE_PVC) {
        Fields F;
        rc = load_fields(h, *c, F);
        if (rc == TMX_OK) {
            if (kind == TMX_FILE_DOMAIN)
                domain_data(fp, F);
            else
                data_pvc(fp, F);
        }
    } else if (kind == TMX_FILE_PRESSURE) {
        rc = pressure_file(fp, h, *c);
    } else {
        rc = mixing_file(fp, h, *c);
    }
    if (std::fclose(fp) != 0 && rc == TMX_OK) rc = fail(TMX_E_INVALID, "error writing %s", path);
    return rc;
}
