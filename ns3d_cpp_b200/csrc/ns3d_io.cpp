// Field I/O in the reference's Tecplot ASCII format (host code).
//
//   write_tecplot_field            (output.cpp:21-87)          -> ns3d_tecplot_write
//   initialize_from_tecplot        (initialization.cpp:35-100) -> ns3d_tecplot_read
//   initialize_from_tecplot_downsample (initialization.cpp:102-198)
//                                                              -> ns3d_tecplot_read_downsample
//
// The format: a TITLE line, a VARIABLES line, a ZONE line (I, J, K =
// nx, ny, nz, DATAPACKING=POINT), then one record "X Y Z rho u v w E p T" per
// cell, x fastest, every value as std::scientific with 8 digits. The writer
// formats with "%.8e", which is what the reference's iostream formatting
// produces, so its files are byte-identical to the reference's for the same
// state; E and T come from the primitives exactly as primitiveToConserved
// computes them. The readers take the records after the ZONE line as a
// whitespace-separated token stream (the reference reads with operator>>);
// E and T are read and dropped, since the reference rebuilds them from the
// primitives right after reading (main.cpp:70-71).
//
// A 256^3 file holds 16.8 M records (~2.6 GB of text), so formatting and
// parsing are split over the host's threads: the writer formats contiguous
// cell ranges into per-thread buffers and writes them in order; the reader
// splits the text at whitespace, counts the tokens of each piece, and parses
// every piece into its place.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ns3d_gpu.h"

namespace {

int host_threads() {
    const unsigned t = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(t, 64u));
}

template <class Fn>
void parallel_ranges(long long n, Fn fn) {
    const int T = (int)std::min<long long>(host_threads(), std::max<long long>(1, n / 4096));
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) {
        const long long a = n * t / T, b = n * (t + 1) / T;
        th.emplace_back([=] { fn(t, a, b); });
    }
    for (auto& x : th) x.join();
}

bool valid_box(const ns3d_params* p) {
    return p && p->global_nx > 0 && p->global_ny > 0 && p->global_nz > 0;
}

// The whole file in memory (binary, so sizes are exact).
bool slurp(const char* path, std::string& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize((size_t)std::max(0LL, size));
    const size_t got = size > 0 ? std::fread(&out[0], 1, (size_t)size, f) : 0;
    std::fclose(f);
    return got == (size_t)std::max(0LL, size);
}

inline bool is_space(char c) {
    return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\v' || c == '\f';
}

// Offset just past the first line starting with "ZONE" (the reference skips
// every line up to and including it), or npos.
size_t after_zone(const std::string& s) {
    size_t pos = 0;
    while (pos < s.size()) {
        size_t eol = s.find('\n', pos);
        if (eol == std::string::npos) eol = s.size();
        if (s.compare(pos, 4, "ZONE") == 0) return eol < s.size() ? eol + 1 : eol;
        pos = eol + 1;
    }
    return std::string::npos;
}

// Parses the first `want` whitespace-separated numbers of s[begin, end) into
// out; returns how many it found (fewer when the text ends early or a token is
// not a number).
long long parse_tokens(const std::string& s, size_t begin, long long want, double* out) {
    const size_t end = s.size();
    const int T = (int)std::min<long long>(host_threads(), std::max<size_t>(1, (end - begin) >> 20));
    // pieces split at whitespace
    std::vector<size_t> cut(T + 1);
    cut[0] = begin;
    cut[T] = end;
    for (int t = 1; t < T; ++t) {
        size_t c = begin + (end - begin) * t / T;
        while (c < end && !is_space(s[c])) ++c;
        cut[t] = std::max(c, cut[t - 1]);
    }
    std::vector<long long> count(T, 0);
    {
        std::vector<std::thread> th;
        for (int t = 0; t < T; ++t)
            th.emplace_back([&, t] {
                long long k = 0;
                bool in = false;
                for (size_t c = cut[t]; c < cut[t + 1]; ++c) {
                    const bool sp = is_space(s[c]);
                    if (!sp && !in) ++k;
                    in = !sp;
                }
                count[t] = k;
            });
        for (auto& x : th) x.join();
    }
    std::vector<long long> first(T + 1, 0);
    for (int t = 0; t < T; ++t) first[t + 1] = first[t] + count[t];
    std::vector<long long> ok(T, 0);
    {
        std::vector<std::thread> th;
        for (int t = 0; t < T; ++t)
            th.emplace_back([&, t] {
                long long idx = first[t];
                const char* c = s.data() + cut[t];
                const char* e = s.data() + cut[t + 1];
                long long good = 0;
                while (idx < want) {
                    while (c < e && is_space(*c)) ++c;
                    if (c >= e) break;
                    char* stop = nullptr;
                    const double v = std::strtod(c, &stop);
                    if (stop == c) break;  // not a number: the stream stops here
                    out[idx++] = v;
                    ++good;
                    c = stop;
                }
                ok[t] = good;
            });
        for (auto& x : th) x.join();
    }
    // tokens are valid up to the first piece that stopped early
    long long n = 0;
    for (int t = 0; t < T; ++t) {
        n += ok[t];
        if (first[t] + ok[t] >= want) return want;
        if (ok[t] < count[t]) break;
    }
    return std::min(n, want);
}

}  // namespace

extern "C" {

ns3d_status ns3d_tecplot_write(const ns3d_params* p, const double* rho, const double* u,
                               const double* v, const double* w, const double* pres,
                               const char* path, double time, int rank) {
    if (!valid_box(p) || !rho || !u || !v || !w || !pres || !path) return NS3D_ERR_INVALID;
    const int nx = p->global_nx, ny = p->global_ny, nz = p->global_nz;
    const long long n = (long long)nx * ny * nz;
    FILE* f = std::fopen(path, "wb");
    if (!f) return NS3D_ERR_FILE;
    std::fprintf(f, "TITLE = \"NS3D Field Rank %d  Time=%.8e\"\n", rank, time);
    std::fprintf(f, "VARIABLES = \"X\" \"Y\" \"Z\" \"rho\" \"u\" \"v\" \"w\" \"E\" \"p\" \"T\"\n");
    std::fprintf(f, "ZONE T=\"rank_%d time=%.8e\" I=%d J=%d K=%d DATAPACKING=POINT\n", rank, time,
                 nx, ny, nz);
    const double gamma = p->gamma, Rgas = p->Rgas;
    const int T = (int)std::min<long long>(host_threads(), std::max<long long>(1, n / 4096));
    // bounded memory: format and write blocks of cells, each block split over the threads
    const long long block = std::max<long long>(1, std::min<long long>(n, (long long)T << 18));
    std::vector<std::string> buf(T);
    for (long long b0 = 0; b0 < n; b0 += block) {
        const long long b1 = std::min(n, b0 + block);
        parallel_ranges(b1 - b0, [&](int t, long long a, long long b) {
            std::string& o = buf[t];
            o.clear();
            char line[256];
            for (long long q = b0 + a; q < b0 + b; ++q) {
                const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / ((long long)nx * ny));
                const double x = p->x0 + i * p->dx, y = p->y0 + j * p->dy, z = p->z0 + k * p->dz;
                // primitiveToConserved (field_structures.h:430-451)
                double rr = rho[q];
                if (rr <= 0.0) rr = 1e-12;
                const double kinetic = 0.5 * (u[q] * u[q] + v[q] * v[q] + w[q] * w[q]);
                const double e_internal = pres[q] / ((gamma - 1.0) * rr);
                const double E = rr * (e_internal + kinetic);
                const double Tq = pres[q] / (rr * Rgas);
                const int len = std::snprintf(line, sizeof line,
                                              "%.8e %.8e %.8e %.8e %.8e %.8e %.8e %.8e %.8e %.8e\n",
                                              x, y, z, rr, u[q], v[q], w[q], E, pres[q], Tq);
                o.append(line, (size_t)len);
            }
        });
        const int used = (int)std::min<long long>(T, std::max<long long>(1, (b1 - b0) / 4096));
        for (int t = 0; t < used; ++t)
            if (std::fwrite(buf[t].data(), 1, buf[t].size(), f) != buf[t].size()) {
                std::fclose(f);
                return NS3D_ERR_FILE;
            }
    }
    return std::fclose(f) == 0 ? NS3D_OK : NS3D_ERR_FILE;
}

ns3d_status ns3d_tecplot_read_downsample(const ns3d_params* p, const char* path, int src_nx,
                                         int src_ny, int src_nz, double* rho, double* u,
                                         double* v, double* w, double* pres) {
    if (!valid_box(p) || !path || !rho || !u || !v || !w || !pres || src_nx <= 0 ||
        src_ny <= 0 || src_nz <= 0)
        return NS3D_ERR_INVALID;
    std::string s;
    if (!slurp(path, s)) {
        std::fprintf(stderr, "Error: cannot open Tecplot file: %s\n", path);
        return NS3D_ERR_FILE;
    }
    const size_t body = after_zone(s);
    const long long nsrc = (long long)src_nx * src_ny * src_nz;
    std::vector<double> rec((size_t)nsrc * 10);
    const long long got = body == std::string::npos ? 0 : parse_tokens(s, body, nsrc * 10, rec.data());
    if (got < nsrc * 10) {
        std::fprintf(stderr, "Error: Tecplot data lines are fewer than expected when reading %s\n",
                     path);
        return NS3D_ERR_FILE;
    }
    const int nx = p->global_nx, ny = p->global_ny, nz = p->global_nz;
    const bool same = nx == src_nx && ny == src_ny && nz == src_nz;
    // nearest source index of initialize_from_tecplot_downsample
    auto map_index = [](int g, int tgt, int src) {
        if (tgt <= 1) return 0;
        const double pos = (double)g * (double)src / (double)tgt;
        return std::clamp((int)std::llround(pos), 0, src - 1);
    };
    const long long n = (long long)nx * ny * nz;
    parallel_ranges(n, [&](int, long long a, long long b) {
        for (long long q = a; q < b; ++q) {
            const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / ((long long)nx * ny));
            const long long sidx =
                same ? q
                     : ((long long)map_index(k, nz, src_nz) * src_ny + map_index(j, ny, src_ny)) * src_nx +
                           map_index(i, nx, src_nx);
            const double* r = &rec[(size_t)sidx * 10];
            rho[q] = r[3];
            u[q] = r[4];
            v[q] = r[5];
            w[q] = r[6];
            pres[q] = r[8];
        }
    });
    return NS3D_OK;
}

ns3d_status ns3d_tecplot_read(const ns3d_params* p, const char* path, double* rho, double* u,
                              double* v, double* w, double* pres) {
    if (!valid_box(p)) return NS3D_ERR_INVALID;
    return ns3d_tecplot_read_downsample(p, path, p->global_nx, p->global_ny, p->global_nz, rho,
                                        u, v, w, pres);
}

ns3d_status ns3d_spectrum_write(const char* path, const double* Ek, int nbins) {
    if (!path || !Ek || nbins < 1) return NS3D_ERR_INVALID;
    FILE* f = std::fopen(path, "wb");
    if (!f) return NS3D_ERR_FILE;
    for (int k = 0; k < nbins; ++k) std::fprintf(f, "%d %g\n", k, Ek[k]);
    return std::fclose(f) == 0 ? NS3D_OK : NS3D_ERR_FILE;
}

ns3d_status ns3d_stats_write(const char* path, double time, const ns3d_turb_stats* s) {
    if (!path || !s) return NS3D_ERR_INVALID;
    FILE* probe = std::fopen(path, "rb");
    const bool exists = probe != nullptr;
    if (probe) std::fclose(probe);
    FILE* f = std::fopen(path, "ab");
    if (!f) return NS3D_ERR_FILE;
    if (!exists)
        std::fprintf(f, "current_time Kinetic Energy TKE u_rms Dissipation Taylor Kol_scale "
                        "Kol_vel Kol_time Taylor_Li Re_lambda Mach_t\n");
    const double v[12] = {time,     s->kinetic_energy, s->tke,     s->u_rms,
                          s->dissipation, s->taylor,   s->eta,     s->u_eta,
                          s->tau_eta, s->taylor_li,    s->re_lambda, s->mach_t};
    for (int q = 0; q < 12; ++q) std::fprintf(f, q < 11 ? "%.8e " : "%.8e\n", v[q]);
    return std::fclose(f) == 0 ? NS3D_OK : NS3D_ERR_FILE;
}

ns3d_status ns3d_residuals_write(const char* path, int step, const double* res, double etot) {
    if (!path || !res) return NS3D_ERR_INVALID;
    // write_residuals_tecplot (output.cpp:92-128): a new file with its header at
    // step 1, one appended row per monitored step after that
    FILE* f = std::fopen(path, step == 1 ? "wb" : "ab");
    if (!f) return NS3D_ERR_FILE;
    if (step == 1) {
        std::fprintf(f, "TITLE = \"Residuals vs Step\"\n");
        std::fprintf(f, "VARIABLES = \"Step\" \"Res_rho\" \"Res_rhou\" \"Res_rhov\" \"Res_rhow\" "
                        "\"Res_E\" \"Etot\"\n");
    }
    std::fprintf(f, "%d %.8e %.8e %.8e %.8e %.8e %.8e\n", step, res[0], res[1], res[2], res[3],
                 res[4], etot);
    return std::fclose(f) == 0 ? NS3D_OK : NS3D_ERR_FILE;
}

ns3d_status ns3d_write_tecplot(ns3d_ctx* ctx, const char* path, double time) {
    if (!ctx || !path) return NS3D_ERR_INVALID;
    ns3d_params p;
    ns3d_status s = ns3d_get_params(ctx, &p);
    if (s != NS3D_OK) return s;
    const size_t n = (size_t)p.global_nx * p.global_ny * p.global_nz;
    std::vector<double> a(5 * n);
    s = ns3d_download_primitive(ctx, &a[0], &a[n], &a[2 * n], &a[3 * n], &a[4 * n], nullptr,
                                nullptr, NS3D_LAYOUT_INTERIOR);
    if (s != NS3D_OK) return s;
    return ns3d_tecplot_write(&p, &a[0], &a[n], &a[2 * n], &a[3 * n], &a[4 * n], path, time, 0);
}

ns3d_status ns3d_read_tecplot(ns3d_ctx* ctx, const char* path) {
    if (!ctx || !path) return NS3D_ERR_INVALID;
    ns3d_params p;
    ns3d_status s = ns3d_get_params(ctx, &p);
    if (s != NS3D_OK) return s;
    const size_t n = (size_t)p.global_nx * p.global_ny * p.global_nz;
    std::vector<double> a(5 * n);
    s = ns3d_tecplot_read(&p, path, &a[0], &a[n], &a[2 * n], &a[3 * n], &a[4 * n]);
    if (s != NS3D_OK) return s;
    return ns3d_upload_primitive(ctx, &a[0], &a[n], &a[2 * n], &a[3 * n], &a[4 * n],
                                 NS3D_LAYOUT_INTERIOR);
}

}  // extern "C"
