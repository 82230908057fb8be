// RBM checkpoints in the reference's on-disk format.
//
// The reference saves `std::unique_ptr<RBM<T>>` with a cereal BinaryOutputArchive
// (Runners/RunRBM.hpp:155-164, files w%04d.dat) and reads it back in
// AbstractRunner::initializeFrom (Runners/AbstractRunner.hpp:83-94).  The bytes
// follow from cereal's binary archive (native byte order, arithmetic types as
// their raw bytes, no names, no header), its unique_ptr wrapper and class
// versioning, SerializeRBM.hpp:20-82 and SerializeEigen.hpp:8-35:
//
//   u8   1                     unique_ptr "valid" (non-null)
//   u32  1                     class version (CEREAL_CLASS_VERSION(RBM<T>, 1)),
//                              written the first time the type appears
//   u8   useBias               bool
//   u32  N, u32 M              getN(), getM()
//   i32  rows = M, i32 cols = N, then W column-major (M x N elements of T)
//   if useBias:
//     i32 N, i32 1, a (N elements);  i32 M, i32 1, b (M elements)
//
// T is std::complex<double>, std::complex<float>, double or float (the element
// type is not recorded in the file; the reader names it).  The machine's FP64
// master parameters are [W column-major | a | b], the same order, so the payload
// is a copy of the masters converted to T.
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.hpp"

namespace yq {

namespace {

size_t elem_size(int elem) {
    switch (elem) {
        case YQ_ARCHIVE_C128: return 16;
        case YQ_ARCHIVE_C64: return 8;
        case YQ_ARCHIVE_F64: return 8;
        case YQ_ARCHIVE_F32: return 4;
        default: throw Error(YQ_E_ARG, "archive: unknown element type");
    }
}

struct Writer {
    std::vector<uint8_t>& out;
    template <typename V>
    void put(V v) {
        const size_t o = out.size();
        out.resize(o + sizeof(V));
        std::memcpy(out.data() + o, &v, sizeof(V));
    }
    void values(int elem, const c128* p, size_t count) {
        for (size_t i = 0; i < count; ++i) {
            const c128 z = p[i];
            switch (elem) {
                case YQ_ARCHIVE_C128: put(z.re); put(z.im); break;
                case YQ_ARCHIVE_C64: put(float(z.re)); put(float(z.im)); break;
                case YQ_ARCHIVE_F64:
                    if (z.im != 0.0) throw Error(YQ_E_ARG, "archive: a real archive needs real parameters");
                    put(z.re);
                    break;
                default:
                    if (z.im != 0.0) throw Error(YQ_E_ARG, "archive: a real archive needs real parameters");
                    put(float(z.re));
                    break;
            }
        }
    }
};

struct Reader {
    const uint8_t* p;
    size_t size, at = 0;
    template <typename V>
    V get() {
        if (size - at < sizeof(V)) throw Error(YQ_E_ARG, "archive: truncated");
        V v;
        std::memcpy(&v, p + at, sizeof(V));
        at += sizeof(V);
        return v;
    }
    void values(int elem, c128* dst, size_t count) {
        if ((size - at) / elem_size(elem) < count) throw Error(YQ_E_ARG, "archive: truncated");
        for (size_t i = 0; i < count; ++i) {
            switch (elem) {
                case YQ_ARCHIVE_C128: {
                    double re = get<double>(), im = get<double>();
                    dst[i] = mk(re, im);
                    break;
                }
                case YQ_ARCHIVE_C64: {
                    float re = get<float>(), im = get<float>();
                    dst[i] = mk(double(re), double(im));
                    break;
                }
                case YQ_ARCHIVE_F64: dst[i] = mk(get<double>(), 0.0); break;
                default: dst[i] = mk(double(get<float>()), 0.0); break;
            }
        }
    }
    // SerializeEigen.hpp:20-35: rows, cols, then the data
    void shape(int rows, int cols, const char* what) {
        const int r = get<int32_t>(), c = get<int32_t>();
        if (r != rows || c != cols)
            throw Error(YQ_E_ARG, std::string("archive: ") + what + " is " + std::to_string(r) + " x " +
                                      std::to_string(c) + ", expected " + std::to_string(rows) + " x " +
                                      std::to_string(cols));
    }
};

}  // namespace

size_t rbm_archive_size(int n, int m, bool bias, int elem) {
    const size_t e = elem_size(elem);
    size_t s = 1 + 4 + 1 + 4 + 4 + 8 + size_t(n) * m * e;
    if (bias) s += 8 + size_t(n) * e + 8 + size_t(m) * e;
    return s;
}

void rbm_archive_shape(const uint8_t* buf, size_t size, int* n, int* m, int* use_bias) {
    Reader r{buf, size};
    if (r.get<uint8_t>() != 1) throw Error(YQ_E_ARG, "archive: null machine pointer");
    (void)r.get<uint32_t>();  // class version: SerializeRBM.hpp's load ignores it
    const uint8_t b = r.get<uint8_t>();
    const uint32_t N = r.get<uint32_t>(), M = r.get<uint32_t>();
    if (N < 1 || M < 1 || N > 65535 || M > 65535) throw Error(YQ_E_ARG, "archive: implausible machine shape");
    *n = int(N);
    *m = int(M);
    *use_bias = b ? 1 : 0;
}

void rbm_archive_write(yq_rbm_s* q, int elem, std::vector<uint8_t>& out) {
    std::vector<c128> p(q->P);
    YQ_CUDA(cudaMemcpyAsync(p.data(), q->p64.p, q->P * sizeof(c128), cudaMemcpyDeviceToHost, q->ctx->stream));
    YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
    out.clear();
    out.reserve(rbm_archive_size(q->n, q->m, q->use_bias, elem));
    Writer w{out};
    w.put(uint8_t(1));
    w.put(uint32_t(1));
    w.put(uint8_t(q->use_bias ? 1 : 0));
    w.put(uint32_t(q->n));
    w.put(uint32_t(q->m));
    const size_t nm = size_t(q->n) * q->m;
    w.put(int32_t(q->m));
    w.put(int32_t(q->n));
    w.values(elem, p.data(), nm);
    if (q->use_bias) {
        w.put(int32_t(q->n));
        w.put(int32_t(1));
        w.values(elem, p.data() + nm, size_t(q->n));
        w.put(int32_t(q->m));
        w.put(int32_t(1));
        w.values(elem, p.data() + nm + q->n, size_t(q->m));
    }
}

void rbm_archive_read(yq_rbm_s* q, int elem, const uint8_t* buf, size_t size) {
    int n = 0, m = 0, bias = 0;
    rbm_archive_shape(buf, size, &n, &m, &bias);
    if (n != q->n || m != q->m || (bias != 0) != q->use_bias)
        throw Error(YQ_E_ARG, "archive: machine shape (N " + std::to_string(n) + ", M " + std::to_string(m) +
                                  ", useBias " + std::to_string(bias) + ") differs from the target machine");
    Reader r{buf, size, 1 + 4 + 1 + 4 + 4};
    std::vector<c128> p(q->P);
    const size_t nm = size_t(n) * m;
    r.shape(m, n, "W");
    r.values(elem, p.data(), nm);
    if (bias) {
        r.shape(n, 1, "a");
        r.values(elem, p.data() + nm, size_t(n));
        r.shape(m, 1, "b");
        r.values(elem, p.data() + nm + n, size_t(m));
    }
    YQ_CUDA(cudaMemcpyAsync(q->p64.p, p.data(), q->P * sizeof(c128), cudaMemcpyHostToDevice, q->ctx->stream));
    YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
    q->version++;
}

std::vector<uint8_t> read_file(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) throw Error(YQ_E_ARG, std::string("archive: cannot open ") + path);
    std::vector<uint8_t> buf;
    uint8_t chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    const bool bad = std::ferror(f) != 0;
    std::fclose(f);
    if (bad) throw Error(YQ_E_ARG, std::string("archive: cannot read ") + path);
    return buf;
}

void write_file(const char* path, const std::vector<uint8_t>& buf) {
    FILE* f = std::fopen(path, "wb");
    if (!f) throw Error(YQ_E_ARG, std::string("archive: cannot create ") + path);
    const size_t put = std::fwrite(buf.data(), 1, buf.size(), f);
    const int closed = std::fclose(f);
    if (put != buf.size() || closed != 0) throw Error(YQ_E_ARG, std::string("archive: cannot write ") + path);
}

}  // namespace yq
