// Recorded raw data: SUPRA's mock metadata formats and int16 frame files, replayed to the device.
//
// Metadata (RxBeamformerParameters::readMetaDataForMock / writeMetaDataForMock,
// Beamformer/RxBeamformerParameters.cpp:93-450):
//   .mock  ASCII: "rawDataMockMetadata v <version>", then numElements, elementLayout x y,
//          numReceivedChannels, numSamples, numTxScanlines, scanlineLayout x y, depth,
//          samplingFrequency, rxNumDepths, speedOfSoundMMperS, the scanlines (x fastest, each in the
//          field order of operator>> for ScanlineRxParameters3D, SupraLib/USImageProperties.cpp:61-82),
//          the depths, the element xs and the element ys. Numbers are read as the reference's stream
//          extraction reads them: doubles with strtod, float fields (depths, element positions) with
//          strtof, integers as unsigned.
//   .json  the object written by writeMetaDataForMock; element positions are read as double then
//          converted to float (jsoncpp asFloat), depths are not stored and are derived as
//          float(depth * i / (rxNumDepths - 1)), as the reference's reader does.
// Frames (UltrasoundInterfaceRawDataMock, SupraLib/InputOutput/UltrasoundInterfaceRawDataMock.cpp:
// 47-204): each data file holds whole int16 frames [tx][channel][sample]; frames play in file order,
// file after file, wrapping to the first file; "streamSequenceOnce" stops after the last frame of the
// last file; "singleImage" repeats the first frame.
//
// B200 replay: a reader thread fills a ring of page-locked host buffers from the files (pread), and
// each sb_mock_reader_next issues one cudaMemcpyAsync of a filled buffer into the caller's device
// buffer on the caller's stream and records an event; the thread refills that buffer only after the
// event, so disk reads, the copy engine and the GPU work on earlier frames overlap.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "supra_b200.h"

using namespace sb;

struct sb_mock_meta {
    uint32_t numElements = 0, elementLayout[2] = {1, 1}, numChannels = 0, numSamples = 0, numTx = 0;
    uint32_t scanlineLayout[2] = {1, 1}, numDepths = 0;
    double depth = 0.0, fs = 0.0, c = 0.0;
    std::vector<sb_scanline_rx> lines;
    std::vector<float> depths, xs, ys;
};

namespace {

// ------------------------------------------------------------------------------------- JSON
struct JVal {
    enum Type { Null, Bool, Num, Str, Arr, Obj } t = Null;
    double num = 0.0;
    bool isInt = false, neg = false;
    uint64_t mag = 0;  // |integer| for integer literals
    bool b = false;
    std::string s;
    std::vector<JVal> arr;
    std::map<std::string, JVal> obj;

    const JVal& operator[](const std::string& k) const {
        static const JVal null;
        auto it = obj.find(k);
        return t == Obj && it != obj.end() ? it->second : null;
    }
    const JVal& operator[](size_t i) const {
        static const JVal null;
        return t == Arr && i < arr.size() ? arr[i] : null;
    }
    double asDouble() const { return t == Num ? num : t == Bool ? (b ? 1.0 : 0.0) : 0.0; }
    float asFloat() const { return static_cast<float>(asDouble()); }
    uint64_t asU64() const {
        if (t != Num) return t == Bool && b ? 1 : 0;
        if (isInt) return neg ? static_cast<uint64_t>(-static_cast<int64_t>(mag)) : mag;
        return num < 0 ? 0 : static_cast<uint64_t>(num);
    }
};

class JsonParser {
public:
    explicit JsonParser(const std::string& s) : m_s(s) {}
    bool parse(JVal& v, std::string* err) {
        bool ok = value(v) && (ws(), m_i == m_s.size());
        if (!ok && err) *err = "JSON syntax error near byte " + std::to_string(m_i);
        return ok;
    }

private:
    void ws() {
        while (m_i < m_s.size()) {
            if (std::isspace(static_cast<unsigned char>(m_s[m_i]))) {
                m_i++;
            } else if (m_s.compare(m_i, 2, "//") == 0) {  // comments (jsoncpp accepts them by default)
                while (m_i < m_s.size() && m_s[m_i] != '\n') m_i++;
            } else if (m_s.compare(m_i, 2, "/*") == 0) {
                const size_t e = m_s.find("*/", m_i + 2);
                m_i = e == std::string::npos ? m_s.size() : e + 2;
            } else {
                break;
            }
        }
    }
    bool lit(const char* w) {
        const size_t n = std::strlen(w);
        if (m_s.compare(m_i, n, w) != 0) return false;
        m_i += n;
        return true;
    }
    bool str(std::string& out) {
        if (m_i >= m_s.size() || m_s[m_i] != '"') return false;
        m_i++;
        while (m_i < m_s.size() && m_s[m_i] != '"') {
            char ch = m_s[m_i++];
            if (ch == '\\' && m_i < m_s.size()) {
                const char e = m_s[m_i++];
                switch (e) {
                case 'n': ch = '\n'; break;
                case 't': ch = '\t'; break;
                case 'r': ch = '\r'; break;
                case 'b': ch = '\b'; break;
                case 'f': ch = '\f'; break;
                case 'u': ch = '?'; m_i = std::min(m_s.size(), m_i + 4); break;  // not used by the format
                default: ch = e;
                }
            }
            out.push_back(ch);
        }
        if (m_i >= m_s.size()) return false;
        m_i++;
        return true;
    }
    bool value(JVal& v) {
        ws();
        if (m_i >= m_s.size()) return false;
        const char ch = m_s[m_i];
        if (ch == '{') {
            v.t = JVal::Obj;
            m_i++;
            ws();
            if (m_i < m_s.size() && m_s[m_i] == '}') return m_i++, true;
            for (;;) {
                ws();
                std::string k;
                if (!str(k)) return false;
                ws();
                if (m_i >= m_s.size() || m_s[m_i] != ':') return false;
                m_i++;
                if (!value(v.obj[k])) return false;
                ws();
                if (m_i < m_s.size() && m_s[m_i] == ',') { m_i++; continue; }
                if (m_i < m_s.size() && m_s[m_i] == '}') return m_i++, true;
                return false;
            }
        }
        if (ch == '[') {
            v.t = JVal::Arr;
            m_i++;
            ws();
            if (m_i < m_s.size() && m_s[m_i] == ']') return m_i++, true;
            for (;;) {
                v.arr.emplace_back();
                if (!value(v.arr.back())) return false;
                ws();
                if (m_i < m_s.size() && m_s[m_i] == ',') { m_i++; continue; }
                if (m_i < m_s.size() && m_s[m_i] == ']') return m_i++, true;
                return false;
            }
        }
        if (ch == '"') {
            v.t = JVal::Str;
            return str(v.s);
        }
        if (lit("true")) { v.t = JVal::Bool; v.b = true; return true; }
        if (lit("false")) { v.t = JVal::Bool; v.b = false; return true; }
        if (lit("null")) { v.t = JVal::Null; return true; }
        // number
        const size_t start = m_i;
        if (m_s[m_i] == '-' || m_s[m_i] == '+') m_i++;
        bool integral = true;
        while (m_i < m_s.size() && (std::isdigit(static_cast<unsigned char>(m_s[m_i])) || std::strchr(".eE+-", m_s[m_i]))) {
            if (std::strchr(".eE", m_s[m_i])) integral = false;
            m_i++;
        }
        if (m_i == start) return false;
        const std::string tok = m_s.substr(start, m_i - start);
        v.t = JVal::Num;
        v.num = std::strtod(tok.c_str(), nullptr);
        if (integral) {
            v.isInt = true;
            v.neg = tok[0] == '-';
            v.mag = std::strtoull(tok.c_str() + (tok[0] == '-' || tok[0] == '+' ? 1 : 0), nullptr, 10);
        }
        return true;
    }

    const std::string& m_s;
    size_t m_i = 0;
};

// ------------------------------------------------------------------------------- ASCII tokens
class Tokens {
public:
    explicit Tokens(std::istream& is) : m_is(is) {}
    bool next(std::string& t) { return static_cast<bool>(m_is >> t); }
    bool d(double& v) { std::string t; return next(t) && num(t, v); }
    bool f(float& v) {
        std::string t;
        if (!next(t)) return false;
        char* e = nullptr;
        errno = 0;
        v = std::strtof(t.c_str(), &e);
        return e && *e == '\0';
    }
    template <typename U> bool u(U& v) {
        std::string t;
        if (!next(t) || t.empty() || t[0] == '-') return false;
        char* e = nullptr;
        const unsigned long long x = std::strtoull(t.c_str(), &e, 10);
        v = static_cast<U>(x);
        return e && *e == '\0';
    }

private:
    static bool num(const std::string& t, double& v) {
        char* e = nullptr;
        v = std::strtod(t.c_str(), &e);
        return e && *e == '\0';
    }
    std::istream& m_is;
};

bool endsWith(const std::string& s, const std::string& suf) {
    return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

int readAscii(const std::string& fn, sb_mock_meta& m) {
    std::ifstream f(fn);
    if (!f.good()) return fail(SB_ERR_INVALID_ARG, "sb_mock_meta_read: cannot open ascii mock file %s", fn.c_str());
    Tokens t(f);
    std::string dummy;
    uint64_t version = 0;
    uint64_t nE, eLx, eLy, nCh, nS, nTx, sLx, sLy, nD;
    if (!t.next(dummy) || !t.next(dummy) || !t.u(version) || !t.u(nE) || !t.u(eLx) || !t.u(eLy) || !t.u(nCh) ||
        !t.u(nS) || !t.u(nTx) || !t.u(sLx) || !t.u(sLy) || !t.d(m.depth) || !t.d(m.fs) || !t.u(nD) || !t.d(m.c))
        return fail(SB_ERR_INVALID_ARG, "sb_mock_meta_read: malformed header in %s", fn.c_str());
    m.numElements = static_cast<uint32_t>(nE);
    m.elementLayout[0] = static_cast<uint32_t>(eLx);
    m.elementLayout[1] = static_cast<uint32_t>(eLy);
    m.numChannels = static_cast<uint32_t>(nCh);
    m.numSamples = static_cast<uint32_t>(nS);
    m.numTx = static_cast<uint32_t>(nTx);
    m.scanlineLayout[0] = static_cast<uint32_t>(sLx);
    m.scanlineLayout[1] = static_cast<uint32_t>(sLy);
    m.numDepths = static_cast<uint32_t>(nD);
    m.lines.assign(static_cast<size_t>(sLx) * sLy, sb_scanline_rx{});
    for (auto& s : m.lines) {  // y outer, x inner: the order of the file
        bool ok = t.d(s.position[0]) && t.d(s.position[1]) && t.d(s.position[2]) && t.d(s.direction[0]) &&
                  t.d(s.direction[1]) && t.d(s.direction[2]) && t.d(s.max_element_distance[0]) &&
                  t.d(s.max_element_distance[1]);
        for (int k = 0; ok && k < 4; k++)
            ok = t.u(s.tx[k].first_active_element[0]) && t.u(s.tx[k].first_active_element[1]) &&
                 t.u(s.tx[k].last_active_element[0]) && t.u(s.tx[k].last_active_element[1]) &&
                 t.u(s.tx[k].tx_scanline_idx) && t.d(s.tx[k].initial_delay_s) && t.d(s.tx_weights[k]);
        if (!ok) return fail(SB_ERR_INVALID_ARG, "sb_mock_meta_read: malformed scanline in %s", fn.c_str());
    }
    m.depths.resize(nD);
    m.xs.resize(nE);
    m.ys.resize(nE);
    for (auto& v : m.depths)
        if (!t.f(v)) return fail(SB_ERR_INVALID_ARG, "sb_mock_meta_read: malformed depths in %s", fn.c_str());
    for (auto& v : m.xs)
        if (!t.f(v)) return fail(SB_ERR_INVALID_ARG, "sb_mock_meta_read: malformed element xs in %s", fn.c_str());
    for (auto& v : m.ys)
        if (!t.f(v)) return fail(SB_ERR_INVALID_ARG, "sb_mock_meta_read: malformed element ys in %s", fn.c_str());
    return SB_OK;
}

int readJson(const std::string& fn, sb_mock_meta& m) {
    std::ifstream f(fn, std::ios::binary);
    if (!f.good()) return fail(SB_ERR_INVALID_ARG, "sb_mock_meta_read: cannot open json mock file %s", fn.c_str());
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    JVal doc;
    std::string err;
    if (!JsonParser(text).parse(doc, &err))
        return fail(SB_ERR_INVALID_ARG, "sb_mock_meta_read: %s: %s", fn.c_str(), err.c_str());
    m.numElements = static_cast<uint32_t>(doc["numElements"].asU64());
    m.numChannels = static_cast<uint32_t>(doc["numReceivedChannels"].asU64());
    m.numSamples = static_cast<uint32_t>(doc["numSamples"].asU64());
    m.numTx = static_cast<uint32_t>(doc["numTxScanlines"].asU64());
    m.scanlineLayout[0] = static_cast<uint32_t>(doc["scanlineLayout"]["x"].asU64());
    m.scanlineLayout[1] = static_cast<uint32_t>(doc["scanlineLayout"]["y"].asU64());
    m.elementLayout[0] = static_cast<uint32_t>(doc["elementLayout"]["x"].asU64());
    m.elementLayout[1] = static_cast<uint32_t>(doc["elementLayout"]["y"].asU64());
    m.depth = doc["depth"].asDouble();
    m.fs = doc["samplingFrequency"].asDouble();
    m.numDepths = static_cast<uint32_t>(doc["rxNumDepths"].asU64());
    m.c = doc["speedOfSoundMMperS"].asDouble();
    const size_t nLines = static_cast<size_t>(m.scanlineLayout[0]) * m.scanlineLayout[1];
    m.lines.assign(nLines, sb_scanline_rx{});
    for (size_t i = 0; i < nLines; i++) {
        const JVal& p = doc["rxScanlines"][i];
        sb_scanline_rx& s = m.lines[i];
        const char* ax[3] = {"x", "y", "z"};
        for (int a = 0; a < 3; a++) {
            s.position[a] = p["position"][ax[a]].asDouble();
            s.direction[a] = p["direction"][ax[a]].asDouble();
        }
        s.max_element_distance[0] = p["maxElementDistance"]["x"].asDouble();
        s.max_element_distance[1] = p["maxElementDistance"]["y"].asDouble();
        for (int k = 0; k < 4; k++) {
            const JVal& tx = p["txParameters"][static_cast<size_t>(k)];
            s.tx[k].first_active_element[0] = static_cast<uint16_t>(tx["firstActiveElementIndex"]["x"].asU64());
            s.tx[k].first_active_element[1] = static_cast<uint16_t>(tx["firstActiveElementIndex"]["y"].asU64());
            s.tx[k].last_active_element[0] = static_cast<uint16_t>(tx["lastActiveElementIndex"]["x"].asU64());
            s.tx[k].last_active_element[1] = static_cast<uint16_t>(tx["lastActiveElementIndex"]["y"].asU64());
            s.tx[k].tx_scanline_idx = static_cast<uint16_t>(tx["txScanlineIdx"].asU64());
            s.tx[k].initial_delay_s = tx["initialDelay"].asDouble();
            s.tx_weights[k] = tx["txWeights"].asDouble();
        }
    }
    m.depths.resize(m.numDepths);
    for (uint32_t i = 0; i < m.numDepths; i++)  // not stored: derived as the reference's reader does
        m.depths[i] = static_cast<float>(m.depth * static_cast<double>(i) / (m.numDepths - 1));
    m.xs.resize(m.numElements);
    m.ys.resize(m.numElements);
    for (uint32_t i = 0; i < m.numElements; i++) {
        m.xs[i] = doc["rxElementPosition"][i]["x"].asFloat();
        m.ys[i] = doc["rxElementPosition"][i]["y"].asFloat();
    }
    return SB_OK;
}

// %.17g with a decimal point kept (the writer's number format for reals)
std::string real(double v) {
    char b[64];
    std::snprintf(b, sizeof(b), "%.17g", v);
    std::string s(b);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return s;
}

}  // namespace

// ------------------------------------------------------------------------------------ reader
struct sb_mock_reader {
    static constexpr int kSlots = 3;
    std::vector<std::string> files;
    std::vector<int> fds;
    std::vector<uint64_t> seqLen;
    uint64_t frameBytes = 0;
    bool singleImage = false, streamOnce = false;
    // producer state
    size_t seq = 0;
    uint64_t frame = 0;
    bool producerDone = false;
    // ring
    void* host[kSlots] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev[kSlots] = {nullptr, nullptr, nullptr};
    bool copyPending[kSlots] = {false, false, false};
    bool filled[kSlots] = {false, false, false};
    bool lastOf[kSlots] = {false, false, false};
    int head = 0, tail = 0;
    bool consumerDone = false;
    std::thread thread;
    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    int error = SB_OK;
    std::string errorMsg;
    int device = 0;

    ~sb_mock_reader() {
        {
            std::lock_guard<std::mutex> l(mu);
            stop = true;
        }
        cv.notify_all();
        if (thread.joinable()) thread.join();
        for (int k = 0; k < kSlots; k++) {
            if (ev[k]) {
                cudaEventSynchronize(ev[k]);
                cudaEventDestroy(ev[k]);
            }
            if (host[k]) cudaFreeHost(host[k]);
        }
        for (int fd : fds)
            if (fd >= 0) close(fd);
    }

    bool readFrame(size_t s, uint64_t i, void* dst, std::string* why) {
        uint64_t off = i * frameBytes, done = 0;
        char* p = static_cast<char*>(dst);
        while (done < frameBytes) {
            const ssize_t r = pread(fds[s], p + done, frameBytes - done, static_cast<off_t>(off + done));
            if (r <= 0) {
                *why = "read of " + files[s] + " failed";
                return false;
            }
            done += static_cast<uint64_t>(r);
        }
        return true;
    }

    // UltrasoundInterfaceRawDataMock::readNextFrame order: the next frame, then advance (and wrap)
    void producer() {
        cudaSetDevice(device);
        for (;;) {
            int slot;
            {
                std::unique_lock<std::mutex> l(mu);
                cv.wait(l, [&] { return stop || (!producerDone && !filled[tail]); });
                if (stop) return;
                slot = tail;
            }
            if (copyPending[slot]) {  // the copy out of this buffer must be complete before it is refilled
                cudaEventSynchronize(ev[slot]);
                copyPending[slot] = false;
            }
            std::string why;
            const bool ok = readFrame(seq, frame, host[slot], &why);
            bool last = false;
            frame = (frame + 1) % seqLen[seq];
            if (frame == 0) {
                seq = (seq + 1) % seqLen.size();
                if (seq == 0 && streamOnce) last = true;
            }
            {
                std::lock_guard<std::mutex> l(mu);
                if (!ok) {
                    error = SB_ERR_INVALID_ARG;
                    errorMsg = why;
                    producerDone = true;
                } else {
                    filled[slot] = true;
                    lastOf[slot] = last;
                    tail = (tail + 1) % kSlots;
                    if (last) producerDone = true;
                }
            }
            cv.notify_all();
        }
    }
};

extern "C" {

int sb_mock_meta_read(const char* filename, sb_mock_meta** out) {
    SB_REQUIRE(filename && out, "sb_mock_meta_read: null argument");
    *out = nullptr;
    auto m = std::make_unique<sb_mock_meta>();
    const std::string fn(filename);
    int st;
    if (endsWith(fn, ".mock")) st = readAscii(fn, *m);
    else if (endsWith(fn, ".json")) st = readJson(fn, *m);
    else return fail(SB_ERR_INVALID_ARG, "sb_mock_meta_read: unknown suffix of %s (.mock or .json)", filename);
    if (st != SB_OK) return st;
    SB_REQUIRE(m->numDepths >= 2 && m->numElements >= 1 && !m->lines.empty(), "sb_mock_meta_read: empty geometry in %s",
               filename);
    *out = m.release();
    return SB_OK;
}

int sb_mock_meta_destroy(sb_mock_meta* meta) {
    delete meta;
    return SB_OK;
}

int sb_mock_meta_geometry(const sb_mock_meta* m, sb_geometry* g, double* depth_mm, double* speed_of_sound_mm_s) {
    SB_REQUIRE(m && g, "sb_mock_meta_geometry: null argument");
    std::memset(g, 0, sizeof(*g));
    g->num_elements = m->numElements;
    g->element_layout[0] = m->elementLayout[0];
    g->element_layout[1] = m->elementLayout[1];
    g->num_channels = m->numChannels;
    g->num_samples = m->numSamples;
    g->num_tx = m->numTx;
    g->rx_layout[0] = m->scanlineLayout[0];
    g->rx_layout[1] = m->scanlineLayout[1];
    g->num_rx = m->scanlineLayout[0] * m->scanlineLayout[1];
    g->num_depths = m->numDepths;
    g->sampling_frequency_hz = m->fs;
    g->element_x_mm = m->xs.data();
    g->element_y_mm = m->ys.data();
    g->depths_mm = m->depths.data();
    g->scanlines = m->lines.data();
    g->element_to_channel = nullptr;
    if (depth_mm) *depth_mm = m->depth;
    if (speed_of_sound_mm_s) *speed_of_sound_mm_s = m->c;
    return SB_OK;
}

int sb_mock_write_json(const char* filename, const sb_geometry* g, double depth_mm, double speed_of_sound_mm_s) {
    SB_REQUIRE(filename && g && g->scanlines && g->element_x_mm && g->element_y_mm, "sb_mock_write_json: null argument");
    std::ofstream f(filename, std::ios::binary);
    SB_REQUIRE(f.good(), "sb_mock_write_json: cannot write %s", filename);
    const char* I1 = "    ";
    const char* I2 = "        ";
    const char* I3 = "            ";
    f << "{\n";
    f << I1 << "\"depth\" : " << real(depth_mm) << ",\n";
    f << I1 << "\"elementLayout\" : { \"x\" : " << g->element_layout[0] << ", \"y\" : " << g->element_layout[1] << " },\n";
    f << I1 << "\"numElements\" : " << g->num_elements << ",\n";
    f << I1 << "\"numReceivedChannels\" : " << g->num_channels << ",\n";
    f << I1 << "\"numSamples\" : " << g->num_samples << ",\n";
    f << I1 << "\"numTxScanlines\" : " << g->num_tx << ",\n";
    f << I1 << "\"rxElementPosition\" : [\n";
    for (uint32_t i = 0; i < g->num_elements; i++)
        f << I2 << "{ \"x\" : " << real(g->element_x_mm[i]) << ", \"y\" : " << real(g->element_y_mm[i]) << " }"
          << (i + 1 < g->num_elements ? ",\n" : "\n");
    f << I1 << "],\n";
    f << I1 << "\"rxNumDepths\" : " << g->num_depths << ",\n";
    f << I1 << "\"rxScanlines\" : [\n";
    for (uint32_t i = 0; i < g->num_rx; i++) {
        const sb_scanline_rx& s = g->scanlines[i];
        f << I2 << "{\n";
        f << I3 << "\"direction\" : { \"x\" : " << real(s.direction[0]) << ", \"y\" : " << real(s.direction[1])
          << ", \"z\" : " << real(s.direction[2]) << " },\n";
        f << I3 << "\"maxElementDistance\" : { \"x\" : " << real(s.max_element_distance[0]) << ", \"y\" : "
          << real(s.max_element_distance[1]) << " },\n";
        f << I3 << "\"position\" : { \"x\" : " << real(s.position[0]) << ", \"y\" : " << real(s.position[1])
          << ", \"z\" : " << real(s.position[2]) << " },\n";
        f << I3 << "\"txParameters\" : [\n";
        for (int k = 0; k < 4; k++) {
            f << I3 << I1 << "{ \"firstActiveElementIndex\" : { \"x\" : " << s.tx[k].first_active_element[0]
              << ", \"y\" : " << s.tx[k].first_active_element[1] << " }, \"initialDelay\" : "
              << real(s.tx[k].initial_delay_s) << ", \"lastActiveElementIndex\" : { \"x\" : "
              << s.tx[k].last_active_element[0] << ", \"y\" : " << s.tx[k].last_active_element[1]
              << " }, \"txScanlineIdx\" : " << s.tx[k].tx_scanline_idx << ", \"txWeights\" : " << real(s.tx_weights[k])
              << " }" << (k < 3 ? ",\n" : "\n");
        }
        f << I3 << "]\n" << I2 << "}" << (i + 1 < g->num_rx ? ",\n" : "\n");
    }
    f << I1 << "],\n";
    f << I1 << "\"samplingFrequency\" : " << real(g->sampling_frequency_hz) << ",\n";
    f << I1 << "\"scanlineLayout\" : { \"x\" : " << g->rx_layout[0] << ", \"y\" : " << g->rx_layout[1] << " },\n";
    f << I1 << "\"speedOfSoundMMperS\" : " << real(speed_of_sound_mm_s) << "\n";
    f << "}\n";
    SB_REQUIRE(f.good(), "sb_mock_write_json: write to %s failed", filename);
    return SB_OK;
}

int sb_mock_reader_create(const sb_mock_meta* meta, const char* data_filenames, int single_image,
                          int stream_sequence_once, sb_mock_reader** out) {
    SB_REQUIRE(meta && data_filenames && out, "sb_mock_reader_create: null argument");
    *out = nullptr;
    auto r = std::make_unique<sb_mock_reader>();
    r->frameBytes = static_cast<uint64_t>(meta->numChannels) * meta->numSamples * meta->numTx * sizeof(int16_t);
    SB_REQUIRE(r->frameBytes > 0, "sb_mock_reader_create: empty frames");
    r->singleImage = single_image != 0;
    r->streamOnce = stream_sequence_once != 0;
    // comma-separated, each name trimmed (the node parameter "mockDataFilename")
    std::stringstream ss(data_filenames);
    std::string item;
    while (std::getline(ss, item, ',')) {
        const size_t a = item.find_first_not_of(" \t\r\n"), b = item.find_last_not_of(" \t\r\n");
        if (a == std::string::npos) continue;
        r->files.push_back(item.substr(a, b - a + 1));
    }
    SB_REQUIRE(!r->files.empty(), "sb_mock_reader_create: no data file named");
    for (const auto& fn : r->files) {
        const int fd = open(fn.c_str(), O_RDONLY);
        r->fds.push_back(fd);
        if (fd < 0) return fail(SB_ERR_INVALID_ARG, "sb_mock_reader_create: cannot open %s", fn.c_str());
        struct stat stt;
        fstat(fd, &stt);
        const uint64_t n = static_cast<uint64_t>(stt.st_size) / r->frameBytes;
        if (n == 0) return fail(SB_ERR_INVALID_ARG, "sb_mock_reader_create: %s holds no whole frame", fn.c_str());
        r->seqLen.push_back(n);
    }
    SB_CUDA(cudaGetDevice(&r->device));
    const int slots = r->singleImage ? 1 : sb_mock_reader::kSlots;
    for (int k = 0; k < slots; k++) {
        SB_CUDA(cudaHostAlloc(&r->host[k], r->frameBytes, cudaHostAllocDefault));
        SB_CUDA(cudaEventCreateWithFlags(&r->ev[k], cudaEventDisableTiming));
    }
    if (r->singleImage) {
        std::string why;
        if (!r->readFrame(0, 0, r->host[0], &why)) return fail(SB_ERR_INVALID_ARG, "sb_mock_reader_create: %s", why.c_str());
    } else {
        sb_mock_reader* p = r.get();
        r->thread = std::thread([p] { p->producer(); });
    }
    *out = r.release();
    return SB_OK;
}

int sb_mock_reader_info(const sb_mock_reader* r, uint64_t* frame_bytes, uint32_t* num_sequences, uint64_t* sequence_lengths) {
    SB_REQUIRE(r, "sb_mock_reader_info: null reader");
    if (frame_bytes) *frame_bytes = r->frameBytes;
    if (num_sequences) *num_sequences = static_cast<uint32_t>(r->seqLen.size());
    if (sequence_lengths)
        for (size_t i = 0; i < r->seqLen.size(); i++) sequence_lengths[i] = r->seqLen[i];
    return SB_OK;
}

int sb_mock_reader_next(sb_mock_reader* r, void* device_frame, sb_stream stream, int* last_frame) {
    SB_REQUIRE(r && device_frame, "sb_mock_reader_next: null argument");
    cudaStream_t st = S(stream);
    if (last_frame) *last_frame = 0;
    if (r->singleImage) {
        SB_CUDA(cudaMemcpyAsync(device_frame, r->host[0], r->frameBytes, cudaMemcpyHostToDevice, st));
        return SB_OK;
    }
    int slot;
    bool last;
    {
        std::unique_lock<std::mutex> l(r->mu);
        SB_REQUIRE(!r->consumerDone, "sb_mock_reader_next: the sequence was streamed once and has ended");
        r->cv.wait(l, [&] { return r->filled[r->head] || (r->producerDone && r->error != SB_OK); });
        if (!r->filled[r->head]) return fail(r->error, "sb_mock_reader_next: %s", r->errorMsg.c_str());
        slot = r->head;
        last = r->lastOf[slot];
    }
    const cudaError_t e = cudaMemcpyAsync(device_frame, r->host[slot], r->frameBytes, cudaMemcpyHostToDevice, st);
    const cudaError_t e2 = e == cudaSuccess ? cudaEventRecord(r->ev[slot], st) : e;
    {
        std::lock_guard<std::mutex> l(r->mu);
        r->copyPending[slot] = e2 == cudaSuccess;
        r->filled[slot] = false;
        r->head = (r->head + 1) % sb_mock_reader::kSlots;
        if (last) r->consumerDone = true;
    }
    r->cv.notify_all();
    if (e2 != cudaSuccess) return cudaFail(e2, "sb_mock_reader_next: copy");
    if (last_frame) *last_frame = last ? 1 : 0;
    return SB_OK;
}

int sb_mock_reader_destroy(sb_mock_reader* r) {
    delete r;
    return SB_OK;
}

}  // extern "C"
