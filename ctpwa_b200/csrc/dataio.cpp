// Event sample readers (see dataio.hpp).
#include "dataio.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>

namespace ctpwa {

namespace {

// Fast whitespace-separated double tokenizer over a whole file.
bool slurp(const std::string& path, std::string& out)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(sz > 0 ? (size_t)sz : 0);
    size_t got = sz > 0 ? std::fread(&out[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    out.resize(got);
    return true;
}

Sample readDat(const std::string& path, int n_final)
{
    std::string buf;
    if (!slurp(path, buf)) throw std::runtime_error("Cannot open file " + path);
    Sample s;
    s.n_final = n_final;
    // Line-oriented like the reference: each non-empty line must begin with
    // four numbers; malformed lines are skipped (reference prints a warning).
    const char* p = buf.c_str();
    const char* end = p + buf.size();
    long lines_ok = 0;
    while (p < end) {
        const char* le = (const char*)std::memchr(p, '\n', (size_t)(end - p));
        if (!le) le = end;
        double v[4];
        const char* q = p;
        int k = 0;
        for (; k < 4; ++k) {
            char* e = nullptr;
            v[k] = std::strtod(q, &e);
            if (e == q || e > le) break;
            q = e;
        }
        if (k == 4) {
            s.p4.insert(s.p4.end(), v, v + 4);
            ++lines_ok;
        }
        p = le + 1;
    }
    s.n = lines_ok / n_final;
    s.p4.resize((size_t)s.n * n_final * 4);  // an incomplete trailing event is dropped
    return s;
}

// numpy .npy reader: little-endian float64, C order, shape (N, n_final, 4).
Sample readNpy(const std::string& path, int n_final)
{
    std::string buf;
    if (!slurp(path, buf)) throw std::runtime_error("Cannot open file " + path);
    if (buf.size() < 10 || std::memcmp(buf.data(), "\x93NUMPY", 6) != 0)
        throw std::runtime_error("not a .npy file: " + path);
    int major = (unsigned char)buf[6];
    size_t hlen, hoff;
    if (major == 1) {
        hlen = (unsigned char)buf[8] | ((size_t)(unsigned char)buf[9] << 8);
        hoff = 10;
    } else {
        hlen = (unsigned char)buf[8] | ((size_t)(unsigned char)buf[9] << 8) | ((size_t)(unsigned char)buf[10] << 16) |
               ((size_t)(unsigned char)buf[11] << 24);
        hoff = 12;
    }
    std::string hdr = buf.substr(hoff, hlen);
    if (hdr.find("'<f8'") == std::string::npos || hdr.find("'fortran_order': False") == std::string::npos)
        throw std::runtime_error(".npy must be C-ordered little-endian float64: " + path);
    size_t data_off = hoff + hlen;
    size_t nbytes = buf.size() - data_off;
    size_t per_event = (size_t)n_final * 4 * sizeof(double);
    Sample s;
    s.n_final = n_final;
    s.n = (long)(nbytes / per_event);
    s.p4.resize((size_t)s.n * n_final * 4);
    std::memcpy(s.p4.data(), buf.data() + data_off, s.p4.size() * sizeof(double));
    return s;
}

}  // namespace

Sample readSample(const std::vector<std::string>& fi, int n_final)
{
    if (fi.size() < 2) throw std::runtime_error("fileinfo must contain at least file type and filename");
    if (fi[0] == "dat") return readDat(fi[1], n_final);
    if (fi[0] == "npy") return readNpy(fi[1], n_final);
    if (fi[0] == "ROOT" || fi[0] == "root")
        throw std::runtime_error("ROOT input is not supported by this build (use dat or npy)");
    throw std::runtime_error("Unknown file type: " + fi[0]);
}

std::vector<double> readWeights(const std::vector<std::string>& fi, long n_events)
{
    std::vector<double> w;
    if (fi.empty()) throw std::runtime_error("weight fileinfo is empty");
    if (fi.size() == 1) {
        w.assign((size_t)n_events, std::stod(fi[0]));
        return w;
    }
    if (fi[0] == "dat") {
        std::string buf;
        if (!slurp(fi[1], buf)) throw std::runtime_error("Cannot open file " + fi[1]);
        const char* p = buf.c_str();
        char* e = nullptr;
        while (true) {
            double v = std::strtod(p, &e);
            if (e == p) break;
            w.push_back(v);
            p = e;
        }
    } else if (fi[0] == "npy") {
        Sample s = readNpy(fi[1], 1);  // reinterpret as flat doubles
        (void)s;
        throw std::runtime_error("npy weights are not supported; use dat");
    } else {
        throw std::runtime_error("Unknown weight file type: " + fi[0]);
    }
    // Size mismatch: pad with zeros / truncate (src/Analysis.cu:400-425)
    w.resize((size_t)n_events, 0.0);
    return w;
}

void shardSample(Sample& s, std::vector<double>& weights, int rank, int world)
{
    if (world < 1 || rank < 0 || rank >= world) throw std::runtime_error("shard: need 0 <= rank < world");
    if (world == 1) return;
    const long lo = (long)((__int128)s.n * rank / world), hi = (long)((__int128)s.n * (rank + 1) / world);
    const size_t stride = (size_t)s.n_final * 4;
    std::vector<double> p(s.p4.begin() + (size_t)lo * stride, s.p4.begin() + (size_t)hi * stride);
    s.p4.swap(p);
    if (!weights.empty()) {
        std::vector<double> w(weights.begin() + lo, weights.begin() + hi);
        weights.swap(w);
    }
    if (!s.weights.empty()) {
        std::vector<double> w(s.weights.begin() + lo, s.weights.begin() + hi);
        s.weights.swap(w);
    }
    s.n = hi - lo;
}

}  // namespace ctpwa
