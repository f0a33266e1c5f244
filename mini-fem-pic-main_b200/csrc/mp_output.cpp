// Asynchronous VTK output from the device buffers: OutputMesh
// (src/meshes.cpp:358-447) and OutputParticles (src/particles.cpp:21-45), the
// reference's ASCII text byte for byte.
//
// The reference formats with std::ostream defaults: doubles as printf's
// "%.6g" (precision 6, general), integers plainly.  std::to_chars with
// chars_format::general and precision 6 is specified as that same conversion
// in the C locale, so the text is identical; it is formatted in parallel
// chunks (one per host thread) that are written in order.
//
// A call snapshots the step's arrays (uh, ef, den; or the particle positions)
// into pinned host buffers with copies on the context's stream, opens the
// file (so an unwritable path fails at once, where the reference exits), and
// returns; a writer thread waits for the copies, formats and writes.  The next
// output call, mp_output_wait and mp_destroy join the writer first.
#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "mp_internal.h"

namespace mp {

struct OutputState {
    // mesh data that does not change between outputs (read from the device once)
    bool have_static = false;
    std::vector<double> node_pos;   // [n_nodes][3]
    std::vector<int> con;           // [n_tets][4]
    std::vector<double> volume;     // [n_tets]
    // the snapshot of one output call
    double *h_uh = nullptr, *h_ef = nullptr, *h_den = nullptr, *h_pos = nullptr;
    size_t pos_cap = 0;
    std::vector<int> node_type;
    cudaEvent_t ready = nullptr;
    std::thread writer;
    int status = MP_OK;
    std::string error;
};

namespace {

inline void put_g(std::string &s, double v) {
    char b[32];
    auto r = std::to_chars(b, b + sizeof b, v, std::chars_format::general, 6);
    s.append(b, r.ptr);
}
inline void put_i(std::string &s, long long v) {
    char b[24];
    auto r = std::to_chars(b, b + sizeof b, v);
    s.append(b, r.ptr);
}

// Formats items [0, n) with fn(i, string&) in parallel chunks and writes
// them in order.
template <class F>
bool write_items(FILE *f, long long n, F fn) {
    if (n <= 0) return true;
    const int hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const int parts = (int)std::min<long long>(hw, (n + 4095) / 4096);
    std::vector<std::string> out(parts);
    auto work = [&](int p) {
        const long long a = n * p / parts, b = n * (p + 1) / parts;
        std::string &s = out[p];
        s.reserve((size_t)(b - a) * 24);
        for (long long i = a; i < b; i++) fn(i, s);
    };
    std::vector<std::thread> th;
    for (int p = 1; p < parts; p++) th.emplace_back(work, p);
    work(0);
    for (auto &t : th) t.join();
    for (auto &s : out)
        if (fwrite(s.data(), 1, s.size(), f) != s.size()) return false;
    return true;
}

bool put(FILE *f, const char *s) { return fputs(s, f) >= 0; }

int write_mesh(OutputState &o, FILE *f, int n_nodes, int n_tets) {
    bool ok = true;
    char line[256];
    ok &= put(f, "<?xml version=\"1.0\"?>\n");
    ok &= put(f, "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    ok &= put(f, "<UnstructuredGrid>\n");
    snprintf(line, sizeof line, "<Piece NumberOfPoints=\"%d\" NumberOfVerts=\"0\" NumberOfLines=\"0\" ", n_nodes);
    ok &= put(f, line);
    snprintf(line, sizeof line, "NumberOfStrips=\"0\" NumberOfCells=\"%d\">\n", n_tets);
    ok &= put(f, line);
    ok &= put(f, "<Points>\n");
    ok &= put(f, "<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    const double *P = o.node_pos.data();
    ok = ok && write_items(f, n_nodes, [&](long long n, std::string &s) {
        put_g(s, P[3 * n]); s += ' '; put_g(s, P[3 * n + 1]); s += ' '; put_g(s, P[3 * n + 2]); s += '\n';
    });
    ok &= put(f, "</DataArray>\n");
    ok &= put(f, "</Points>\n");
    ok &= put(f, "<Cells>\n");
    ok &= put(f, "<DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n");
    const int *Cn = o.con.data();
    ok = ok && write_items(f, n_tets, [&](long long e, std::string &s) {
        for (int v = 0; v < 4; v++) {
            put_i(s, Cn[4 * e + v]);
            s += v < 3 ? ' ' : '\n';
        }
    });
    ok &= put(f, "</DataArray>\n");
    ok &= put(f, "<DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n");
    ok = ok && write_items(f, n_tets, [&](long long e, std::string &s) { put_i(s, (e + 1) * 4); s += ' '; });
    ok &= put(f, "\n</DataArray>\n");
    ok &= put(f, "<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n");
    ok = ok && write_items(f, n_tets, [&](long long, std::string &s) { s += "10 "; });
    ok &= put(f, "\n</DataArray>\n");
    ok &= put(f, "</Cells>\n");
    ok &= put(f, "<PointData Scalars=\"phi\">\n");
    ok &= put(f, "<DataArray type=\"Int32\" Name=\"node_index\" format=\"ascii\">\n");
    ok = ok && write_items(f, n_nodes, [&](long long n, std::string &s) { put_i(s, n); s += ' '; });
    ok &= put(f, "\n</DataArray>\n");
    ok &= put(f, "<DataArray type=\"Int32\" Name=\"node_type\" format=\"ascii\">\n");
    const int *T = o.node_type.data();
    ok = ok && write_items(f, n_nodes, [&](long long n, std::string &s) { put_i(s, T[n]); s += ' '; });
    ok &= put(f, "\n</DataArray>\n");
    ok &= put(f, "<DataArray type=\"Float32\" Name=\"phi\" format=\"ascii\">\n");
    ok = ok && write_items(f, n_nodes, [&](long long n, std::string &s) { put_g(s, o.h_uh[n]); s += ' '; });
    ok &= put(f, "\n</DataArray>\n");
    ok &= put(f, "<DataArray type=\"Float32\" Name=\"ion_den\" format=\"ascii\">\n");
    ok = ok && write_items(f, n_nodes, [&](long long n, std::string &s) { put_g(s, o.h_den[n]); s += ' '; });
    ok &= put(f, "\n</DataArray>\n");
    ok &= put(f, "</PointData>\n");
    ok &= put(f, "<CellData Vectors=\"ef\">\n");
    ok &= put(f, "<DataArray type=\"Float32\" NumberOfComponents=\"3\" Name=\"ef\" format=\"ascii\">\n");
    ok = ok && write_items(f, n_tets, [&](long long e, std::string &s) {
        put_g(s, o.h_ef[3 * e]); s += ' '; put_g(s, o.h_ef[3 * e + 1]); s += ' '; put_g(s, o.h_ef[3 * e + 2]);
        s += ' ';
    });
    ok &= put(f, "\n</DataArray>\n");
    ok &= put(f, "<DataArray type=\"Float32\" Name=\"cell_volume\" format=\"ascii\">\n");
    const double *V = o.volume.data();
    ok = ok && write_items(f, n_tets, [&](long long e, std::string &s) { put_g(s, V[e]); s += ' '; });
    ok &= put(f, "\n</DataArray>\n");
    ok &= put(f, "</CellData>\n");
    ok &= put(f, "</Piece>\n");
    ok &= put(f, "</UnstructuredGrid>\n");
    ok &= put(f, "</VTKFile>\n");
    return ok ? MP_OK : MP_ERR_ARG;
}

int write_particles(OutputState &o, FILE *f, long long n) {
    bool ok = true;
    char line[256];
    ok &= put(f, "<?xml version=\"1.0\"?>\n");
    ok &= put(f, "<VTKFile type=\"PolyData\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    ok &= put(f, "<PolyData>\n");
    snprintf(line, sizeof line, "<Piece NumberOfPoints=\"%lld\" NumberOfVerts=\"0\" NumberOfLines=\"0\" ", n);
    ok &= put(f, line);
    ok &= put(f, "NumberOfStrips=\"0\" NumberOfCells=\"0\">\n");
    ok &= put(f, "<Points>\n");
    ok &= put(f, "<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    const double *P = o.h_pos;  // [n][3]
    ok = ok && write_items(f, n, [&](long long i, std::string &s) {
        put_g(s, P[3 * i]); s += ' '; put_g(s, P[3 * i + 1]); s += ' '; put_g(s, P[3 * i + 2]); s += '\n';
    });
    ok &= put(f, "</DataArray>\n");
    ok &= put(f, "</Points>\n");
    ok &= put(f, "</Piece>\n");
    ok &= put(f, "</PolyData>\n");
    ok &= put(f, "</VTKFile>\n");
    return ok ? MP_OK : MP_ERR_ARG;
}

OutputState *state(mp_ctx *ctx) {
    if (!ctx->output) ctx->output = new OutputState();
    return static_cast<OutputState *>(ctx->output);
}

int join(mp_ctx *ctx) {
    if (!ctx->output) return MP_OK;
    OutputState &o = *static_cast<OutputState *>(ctx->output);
    if (o.writer.joinable()) o.writer.join();
    int rc = o.status;
    if (rc) fail(ctx, rc, o.error);
    o.status = MP_OK;
    return rc;
}

int load_static(mp_ctx *ctx, OutputState &o) {
    if (o.have_static) return MP_OK;
    const int nn = ctx->n_nodes, nt = ctx->n_tets;
    o.node_pos.resize(3 * (size_t)nn);
    o.con.resize(4 * (size_t)nt);
    o.volume.resize(nt);
    std::vector<TetRec> rec(nt);
    MP_CUDA(ctx, cudaMemcpyAsync(o.node_pos.data(), ctx->node_pos, sizeof(double) * 3 * nn, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(o.con.data(), ctx->con, sizeof(int) * 4 * nt, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(rec.data(), ctx->tets, sizeof(TetRec) * nt, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int e = 0; e < nt; e++) o.volume[e] = rec[e].volume;
    if (!o.ready) MP_CUDA(ctx, cudaEventCreateWithFlags(&o.ready, cudaEventDisableTiming));
    o.have_static = true;
    return MP_OK;
}

}  // namespace

void output_free(mp_ctx *ctx) {
    if (!ctx->output) return;
    OutputState *o = static_cast<OutputState *>(ctx->output);
    if (o->writer.joinable()) o->writer.join();
    double *pinned[] = {o->h_uh, o->h_ef, o->h_den, o->h_pos};
    for (double *p : pinned)
        if (p) cudaFreeHost(p);
    if (o->ready) cudaEventDestroy(o->ready);
    delete o;
    ctx->output = nullptr;
}

}  // namespace mp

using namespace mp;

int mp_output_mesh(mp_ctx *ctx, int32_t ts, const char *dir, const int32_t *node_type, int64_t node_type_stride) {
    if (!ctx || !node_type || node_type_stride < (int64_t)sizeof(int32_t)) return MP_ERR_ARG;
    if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup: uh and ef are not defined");
    int rc = join(ctx);
    if (rc) return rc;
    OutputState &o = *state(ctx);
    if ((rc = load_static(ctx, o))) return rc;
    const int nn = ctx->n_nodes, nt = ctx->n_tets;
    if (!o.h_uh) {
        MP_CUDA(ctx, cudaHostAlloc(&o.h_uh, sizeof(double) * nn, 0));
        MP_CUDA(ctx, cudaHostAlloc(&o.h_den, sizeof(double) * nn, 0));
        MP_CUDA(ctx, cudaHostAlloc(&o.h_ef, sizeof(double) * 3 * nt, 0));
    }
    o.node_type.resize(nn);
    const char *tb = reinterpret_cast<const char *>(node_type);
    for (int n = 0; n < nn; n++) std::memcpy(&o.node_type[n], tb + n * node_type_stride, sizeof(int32_t));
    char name[64];
    snprintf(name, sizeof name, "mesh_%04d.vtu", ts + 1);  // setfill('0') << setw(4) << ts+1
    std::string path = dir && *dir ? std::string(dir) + "/" + name : std::string(name);
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return fail(ctx, MP_ERR_ARG, "Failed to open file " + path);
    MP_CUDA(ctx, cudaMemcpyAsync(o.h_uh, ctx->uh, sizeof(double) * nn, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(o.h_den, ctx->den, sizeof(double) * nn, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(o.h_ef, ctx->ef, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaEventRecord(o.ready, ctx->stream));
    OutputState *op = &o;
    o.writer = std::thread([op, f, nn, nt, path] {
        int st = cudaEventSynchronize(op->ready) == cudaSuccess ? write_mesh(*op, f, nn, nt) : MP_ERR_CUDA;
        if (fclose(f) != 0 && st == MP_OK) st = MP_ERR_ARG;
        if (st) {
            op->status = st;
            op->error = "writing " + path + " failed";
        }
    });
    return MP_OK;
}

int mp_output_particles(mp_ctx *ctx, const char *path) {
    if (!ctx || !path || !*path) return MP_ERR_ARG;
    int rc = join(ctx);
    if (rc) return rc;
    OutputState &o = *state(ctx);
    if ((rc = load_static(ctx, o))) return rc;
    int64_t n = 0;
    if ((rc = mp_particles_count(ctx, &n))) return rc;
    if ((size_t)n > o.pos_cap) {
        if (o.h_pos) cudaFreeHost(o.h_pos);
        o.h_pos = nullptr;
        o.pos_cap = 0;
        MP_CUDA(ctx, cudaHostAlloc(&o.h_pos, sizeof(double) * 3 * std::max<int64_t>(1, n), 0));
        o.pos_cap = (size_t)std::max<int64_t>(1, n);
    }
    FILE *f = fopen(path, "wb");
    if (!f) return fail(ctx, MP_ERR_ARG, std::string("Failed to open output file ") + path);
    // the reference's particle order (the live particles by id)
    if (n > 0) {
        rc = mp_particles_download(ctx, n, o.h_pos, 3 * sizeof(double), nullptr, 0, nullptr, 0, nullptr, 0, nullptr,
                                   MP_ORDER_ID);
        if (rc) {
            fclose(f);
            return rc;
        }
    }
    OutputState *op = &o;
    std::string p(path);
    o.writer = std::thread([op, f, n, p] {
        int st = write_particles(*op, f, n);
        if (fclose(f) != 0 && st == MP_OK) st = MP_ERR_ARG;
        if (st) {
            op->status = st;
            op->error = "writing " + p + " failed";
        }
    });
    return MP_OK;
}

int mp_output_wait(mp_ctx *ctx) {
    if (!ctx) return MP_ERR_ARG;
    return join(ctx);
}
