// VTU output: the reference's inline-XML UnstructuredGrid writers
// (crates/solvix-io/src/vtu.rs), byte for byte.
//
// The ASCII form (vtu.rs:14-115, write_vtu_ex) prints every f64 as Rust's
// `{}` Display does: the shortest digits that read back to the same bits
// (std::to_chars' shortest scientific form supplies them with their decimal
// exponent), laid out positionally with zeros (never an exponent), "-0"
// for negative zero, "NaN" and "inf" / "-inf".  The reference
// builds the file in one String on one thread; here the per-node and
// per-element lines are formatted in contiguous chunks on the host cores and
// concatenated in order, so the bytes do not depend on the thread count.
//
// The binary form (vtu.rs:148-288, write_vtu_binary) writes the six arrays
// as little-endian raw blocks after the XML, each preceded by its Int32
// byte count, with the XML offsets pointing into that appended stream.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "solvix_gpu.h"
#include "svx_text.h"

namespace {

void put_f64(std::string& out, double v) { svx::rust_display_f64(out, v); }

void put_u64(std::string& out, unsigned long long v) {
    char buf[24];
    const auto r = std::to_chars(buf, buf + sizeof buf, v);
    out.append(buf, r.ptr);
}

// VTK cell types of vtu.rs:62-70 / :181-189, indexed by svx_elem_kind.
long long vtk_type(int kind) {
    static const long long t[8] = {5, 9, 23, 9, 23, 12, 10, 3};
    return (kind >= 0 && kind < 8) ? t[kind] : 0;
}

// The file as a list of pieces written in order (chunks move in, nothing
// is concatenated).
struct Pieces {
    std::vector<std::string> parts{std::string()};
    std::string& tail() { return parts.back(); }
    Pieces& operator+=(const char* t) {
        tail() += t;
        return *this;
    }
    Pieces& operator+=(const std::string& t) {
        tail() += t;
        return *this;
    }
};

// fn(i, out) for i in [0, count), formatted in contiguous chunks on up to
// `threads` host threads and appended to `dst` in index order.
template <class F>
void format_rows(Pieces& dst, int64_t count, int threads, F&& fn) {
    if (count <= 0) return;
    const int64_t min_chunk = 4096;
    int chunks = int(std::min<int64_t>(std::max(1, threads) * 4,
                                       (count + min_chunk - 1) / min_chunk));
    chunks = std::max(chunks, 1);
    std::vector<std::string> parts(static_cast<size_t>(chunks));
    std::atomic<int> next{0};
    auto work = [&] {
        for (int c = next.fetch_add(1); c < chunks; c = next.fetch_add(1)) {
            const int64_t a = count * c / chunks, b = count * (c + 1) / chunks;
            std::string& s = parts[size_t(c)];
            s.reserve(size_t(b - a) * 48);
            for (int64_t i = a; i < b; ++i) fn(i, s);
        }
    };
    const int n_threads = std::min(threads, chunks);
    std::vector<std::thread> pool;
    for (int t = 1; t < n_threads; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (auto& p : parts) dst.parts.push_back(std::move(p));
    dst.parts.emplace_back();
}

void set_error(svx_error_t* err, int code, const std::string& msg) {
    if (!err) return;
    std::memset(err, 0, sizeof(*err));
    err->code = code;
    err->elem_index = -1;
    std::snprintf(err->message, sizeof(err->message), "%s", msg.c_str());
}

int write_file(const char* path, const std::vector<std::pair<const char*, size_t>>& spans,
               svx_error_t* err) {
    std::FILE* f = std::fopen(path, "wb");
    if (!f) {
        set_error(err, SVX_IO_ERROR, std::string("could not create ") + path + ": " +
                                         std::strerror(errno));
        return SVX_IO_ERROR;
    }
    bool ok = true;
    for (const auto& sp : spans)
        if (sp.second && std::fwrite(sp.first, 1, sp.second, f) != sp.second) ok = false;
    const int closed = std::fclose(f);
    if (!ok || closed != 0) {
        set_error(err, SVX_IO_ERROR, std::string("could not write ") + path);
        return SVX_IO_ERROR;
    }
    set_error(err, SVX_OK, "");
    return SVX_OK;
}

int write_ascii(const char* path, const svx_vtu_data_t* d, int threads, svx_error_t* err) {
    const int64_t nn = d->n_nodes, ne = d->n_elem;
    Pieces s;
    s += "<?xml version=\"1.0\"?>\n";
    s += "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_format=\"ascii\">\n";
    s += "  <UnstructuredGrid>\n";
    s += "    <Piece NumberOfPoints=\"";
    put_u64(s.tail(), (unsigned long long)nn);
    s += "\" NumberOfCells=\"";
    put_u64(s.tail(), (unsigned long long)ne);
    s += "\">\n";
    s += "      <Points>\n";
    s += "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    format_rows(s, nn, threads, [&](int64_t i, std::string& o) {
        o += "          ";
        put_f64(o, d->xyz[3 * i]);
        o += ' ';
        put_f64(o, d->xyz[3 * i + 1]);
        o += ' ';
        put_f64(o, d->xyz[3 * i + 2]);
        o += '\n';
    });
    s += "        </DataArray>\n      </Points>\n";
    s += "      <Cells>\n";
    s += "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n          ";
    format_rows(s, ne, threads, [&](int64_t e, std::string& o) {
        for (int64_t q = d->conn_ptr[e]; q < d->conn_ptr[e + 1]; ++q) {
            put_u64(o, (unsigned long long)d->conn[q]);
            o += ' ';
        }
    });
    s += "\n        </DataArray>\n";
    s += "        <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n          ";
    format_rows(s, ne, threads, [&](int64_t e, std::string& o) {
        put_u64(o, (unsigned long long)(d->conn_ptr[e + 1] - d->conn_ptr[0]));
        o += ' ';
    });
    s += "\n        </DataArray>\n";
    s += "        <DataArray type=\"Int64\" Name=\"types\" format=\"ascii\">\n          ";
    format_rows(s, ne, threads, [&](int64_t e, std::string& o) {
        put_u64(o, (unsigned long long)vtk_type(d->kind[e]));
        o += ' ';
    });
    s += "\n        </DataArray>\n      </Cells>\n";
    s += "      <PointData>\n        <DataArray type=\"Float64\" Name=\"Displacement\" "
         "NumberOfComponents=\"3\" format=\"ascii\">\n";
    format_rows(s, nn, threads, [&](int64_t i, std::string& o) {
        const bool has = i < d->n_disp;
        o += "          ";
        put_f64(o, has ? d->displacements[3 * i] : 0.0);
        o += ' ';
        put_f64(o, has ? d->displacements[3 * i + 1] : 0.0);
        o += ' ';
        put_f64(o, has ? d->displacements[3 * i + 2] : 0.0);
        o += '\n';
    });
    s += "        </DataArray>\n      </PointData>\n";
    for (int32_t a = 0; a < d->n_extra; ++a) {
        s += "      <PointData>\n        <DataArray type=\"Float64\" Name=\"";
        s += d->extra_names[a];
        s += "\" format=\"ascii\">\n";
        const double* v = d->extra_values[a];
        const int64_t len = d->extra_len[a];
        format_rows(s, nn, threads, [&](int64_t i, std::string& o) {
            o += "          ";
            put_f64(o, i < len ? v[i] : 0.0);
            o += '\n';
        });
        s += "        </DataArray>\n      </PointData>\n";
    }
    s += "      <CellData>\n        <DataArray type=\"Float64\" Name=\"VonMises\" "
         "format=\"ascii\">\n";
    format_rows(s, ne, threads, [&](int64_t e, std::string& o) {
        o += "          ";
        put_f64(o, e < d->n_von_mises ? d->von_mises[e] : 0.0);
        o += '\n';
    });
    s += "        </DataArray>\n      </CellData>\n";
    s += "    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n";
    std::vector<std::pair<const char*, size_t>> spans;
    for (const auto& p : s.parts) spans.emplace_back(p.data(), p.size());
    return write_file(path, spans, err);
}

// little-endian raw bytes of one value (the host is little-endian)
template <class T>
void put_le(std::vector<char>& out, T v) {
    static_assert(sizeof(T) == 8 || sizeof(T) == 4, "8- or 4-byte values");
    char b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));
    out.insert(out.end(), b, b + sizeof(T));
}

int write_binary(const char* path, const svx_vtu_data_t* d, svx_error_t* err) {
    const int64_t nn = d->n_nodes, ne = d->n_elem;
    std::vector<char> blob;
    std::vector<size_t> offs;
    // AppendedData::append (vtu.rs:130-141): Int32 byte count, then the block
    auto append = [&](const std::vector<char>& block) -> bool {
        if (block.size() > size_t(INT32_MAX)) return false;
        offs.push_back(blob.size());
        put_le<int32_t>(blob, int32_t(block.size()));
        blob.insert(blob.end(), block.begin(), block.end());
        return true;
    };
    std::vector<char> points, conn, offsets, types, disp, vm;
    points.reserve(size_t(nn) * 24);
    for (int64_t i = 0; i < 3 * nn; ++i) put_le<double>(points, d->xyz[i]);
    const int64_t nc = ne > 0 ? d->conn_ptr[ne] - d->conn_ptr[0] : 0;
    conn.reserve(size_t(nc) * 8);
    for (int64_t q = d->conn_ptr[0]; ne > 0 && q < d->conn_ptr[ne]; ++q)
        put_le<int64_t>(conn, int64_t(d->conn[q]));
    offsets.reserve(size_t(ne) * 8);
    types.reserve(size_t(ne) * 8);
    for (int64_t e = 0; e < ne; ++e) {
        put_le<int64_t>(offsets, d->conn_ptr[e + 1] - d->conn_ptr[0]);
        put_le<int64_t>(types, vtk_type(d->kind[e]));
    }
    disp.reserve(size_t(nn) * 24);
    for (int64_t i = 0; i < nn; ++i)
        for (int c = 0; c < 3; ++c)
            put_le<double>(disp, i < d->n_disp ? d->displacements[3 * i + c] : 0.0);
    vm.reserve(size_t(ne) * 8);
    for (int64_t e = 0; e < ne; ++e)
        put_le<double>(vm, e < d->n_von_mises ? d->von_mises[e] : 0.0);
    for (const auto* b : {&points, &conn, &offsets, &types, &disp, &vm})
        if (!append(*b)) {
            set_error(err, SVX_IO_ERROR,
                      "VTK appended-data block exceeds the Int32 byte-count header");
            return SVX_IO_ERROR;
        }
    std::string x;
    x += "<?xml version=\"1.0\"?>\n"
         "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
         "  <UnstructuredGrid>\n";
    x += "    <Piece NumberOfPoints=\"";
    put_u64(x, (unsigned long long)nn);
    x += "\" NumberOfCells=\"";
    put_u64(x, (unsigned long long)ne);
    x += "\">\n";
    auto off = [&](int k) {
        std::string t;
        put_u64(t, (unsigned long long)offs[size_t(k)]);
        return t;
    };
    x += "      <Points>\n        <DataArray type=\"Float64\" NumberOfComponents=\"3\" "
         "format=\"appended\" offset=\"" + off(0) + "\"/>\n      </Points>\n";
    x += "      <Cells>\n        <DataArray type=\"Int64\" Name=\"connectivity\" "
         "format=\"appended\" offset=\"" + off(1) + "\"/>\n";
    x += "        <DataArray type=\"Int64\" Name=\"offsets\" format=\"appended\" offset=\"" +
         off(2) + "\"/>\n";
    x += "        <DataArray type=\"Int64\" Name=\"types\" format=\"appended\" offset=\"" +
         off(3) + "\"/>\n      </Cells>\n";
    x += "      <PointData>\n        <DataArray type=\"Float64\" Name=\"Displacement\" "
         "NumberOfComponents=\"3\" format=\"appended\" offset=\"" + off(4) +
         "\"/>\n      </PointData>\n";
    x += "      <CellData>\n        <DataArray type=\"Float64\" Name=\"VonMises\" "
         "format=\"appended\" offset=\"" + off(5) + "\"/>\n      </CellData>\n";
    x += "    </Piece>\n  </UnstructuredGrid>\n  <AppendedData encoding=\"raw\">_";
    static const char tail[] = "\n  </AppendedData>\n</VTKFile>\n";
    return write_file(path, {{x.data(), x.size()}, {blob.data(), blob.size()},
                             {tail, sizeof(tail) - 1}},
                      err);
}

}  // namespace

extern "C" int svx_write_vtu(const char* path, const svx_vtu_data_t* d, int32_t binary,
                             int32_t threads, svx_error_t* err) {
    if (!path || !d) {
        set_error(err, SVX_BAD_ARGUMENT, "null argument");
        return SVX_BAD_ARGUMENT;
    }
    auto bad = [&](const std::string& msg) {
        set_error(err, SVX_BAD_ARGUMENT, msg);
        return SVX_BAD_ARGUMENT;
    };
    if (d->n_nodes < 0 || d->n_elem < 0 || d->n_disp < 0 || d->n_von_mises < 0 || d->n_extra < 0)
        return bad("negative size");
    if (d->n_nodes > 0 && !d->xyz) return bad("null xyz");
    if (d->n_elem > 0 && (!d->kind || !d->conn_ptr || !d->conn)) return bad("null element array");
    if (d->n_disp > 0 && !d->displacements) return bad("null displacements");
    if (d->n_von_mises > 0 && !d->von_mises) return bad("null von Mises");
    if (d->n_extra > 0 && (!d->extra_names || !d->extra_values || !d->extra_len))
        return bad("null extra arrays");
    if (binary && d->n_extra > 0) return bad("extra arrays are written by the ASCII form only");
    for (int64_t e = 0; e < d->n_elem; ++e) {
        if (d->conn_ptr[e + 1] < d->conn_ptr[e]) return bad("conn_ptr must not decrease");
        for (int64_t q = d->conn_ptr[e]; q < d->conn_ptr[e + 1]; ++q)
            if (d->conn[q] < 0 || d->conn[q] >= d->n_nodes)
                return bad("connectivity index out of range");
    }
    for (int32_t a = 0; a < d->n_extra; ++a)
        if (!d->extra_names[a] || (d->extra_len[a] > 0 && !d->extra_values[a]))
            return bad("null extra array");
    int t = threads;
    if (t <= 0) t = int(std::max(1u, std::thread::hardware_concurrency()));
    try {
        return binary ? write_binary(path, d, err) : write_ascii(path, d, t, err);
    } catch (const std::bad_alloc&) {
        set_error(err, SVX_OOM, "host allocation failed");
        return SVX_OOM;
    }
}
