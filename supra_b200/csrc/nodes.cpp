// Node layer: SUPRA's receive-path nodes re-hosted on the C ABI (declarations and the interface
// contract in include/supra_b200_nodes.hpp), plus the C entry points sb_node_* / sb_graph_*.
//
// Parameter tables follow the reference constructors: BeamformingNode.cpp:42-49,
// RawDelayNode.cpp:43-47, BeamformingMVNode.cpp:42-46, HilbertFirEnvelopeNode.cpp:42-43,
// IQDemodulatorNode.cpp:52-71 (constants :26-29), LogCompressorNode.cpp:42-45,
// ScanConverterNode.cpp:41-43.
#include <cuda_runtime.h>

#include <algorithm>
#include <deque>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <sstream>

#include "supra_b200.h"
#include "supra_b200_nodes.hpp"

namespace sb {
void setError(const char* fmt, ...);  // thread-local message behind sb_last_error() (core.cu)
}

namespace supra_b200 {

// ------------------------------------------------------------------------------------ types

const char* dataTypeName(DataType t) {
    switch (t) {
    case DataType::Int16: return "int16";
    case DataType::Float: return "float";
    case DataType::Uint8: return "uint8";
    case DataType::Complex64: return "complex64";
    case DataType::Uint16: return "uint16";
    }
    return "?";
}

bool parseDataType(const std::string& s, DataType& t) {
    if (s == "int16" || s == "int16_t") t = DataType::Int16;
    else if (s == "float") t = DataType::Float;
    else if (s == "uint8" || s == "uint8_t") t = DataType::Uint8;
    else if (s == "uint16" || s == "uint16_t") t = DataType::Uint16;
    else if (s == "complex64") t = DataType::Complex64;
    else return false;
    return true;
}

static size_t dtypeBytes(DataType t) {
    switch (t) {
    case DataType::Int16: return 2;
    case DataType::Float: return 4;
    case DataType::Uint8: return 1;
    case DataType::Complex64: return 8;
    case DataType::Uint16: return 2;
    }
    return 0;
}

static std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) a++;
    while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) b--;
    return s.substr(a, b - a);
}

static std::string fmtDouble(double v) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.15g", v);
    return buf;
}

// ------------------------------------------------------------------------- dictionaries

void ValueRangeDictionary::setRange(const std::string& name, const std::string& type, double min, double max,
                                    const std::string& def, const std::string& label) {
    ParamSpec s;
    s.name = name;
    s.type = type;
    s.label = label;
    s.defaultValue = def;
    s.isRange = true;
    s.min = min;
    s.max = max;
    m_specs.push_back(s);
}

void ValueRangeDictionary::setChoices(const std::string& name, const std::string& type,
                                      const std::vector<std::string>& choices, const std::string& def,
                                      const std::string& label) {
    ParamSpec s;
    s.name = name;
    s.type = type;
    s.label = label;
    s.defaultValue = def;
    s.choices = choices;
    m_specs.push_back(s);
}

const ParamSpec* ValueRangeDictionary::find(const std::string& name) const {
    for (const ParamSpec& s : m_specs)
        if (s.name == name) return &s;
    return nullptr;
}

static bool parseBool(const std::string& v, bool& b) {
    std::string l = v;
    std::transform(l.begin(), l.end(), l.begin(), [](unsigned char c) { return std::tolower(c); });
    if (l == "true" || l == "1") b = true;
    else if (l == "false" || l == "0") b = false;
    else return false;
    return true;
}

// Canonical form of a value of the spec's type, or "" if it does not parse or is out of range.
static std::string canonical(const ParamSpec& spec, const std::string& raw) {
    const std::string v = trim(raw);
    if (spec.type == "double" || spec.type == "uint32_t" || spec.type == "int32_t") {
        char* end = nullptr;
        const double d = std::strtod(v.c_str(), &end);
        if (v.empty() || end == v.c_str() || *end != '\0' || !std::isfinite(d)) return "";
        if (spec.type != "double" && d != std::floor(d)) return "";
        if (spec.type == "uint32_t" && d < 0) return "";
        if (spec.isRange && (d < spec.min || d > spec.max)) return "";
        return spec.type == "double" ? fmtDouble(d) : std::to_string(static_cast<long long>(d));
    }
    if (spec.type == "bool") {
        bool b;
        if (!parseBool(v, b)) return "";
        return b ? "true" : "false";
    }
    if (spec.type == "DataType") {
        DataType t;
        if (!parseDataType(v, t)) return "";
        const std::string n = dataTypeName(t);
        for (const std::string& c : spec.choices)
            if (c == n) return n;
        return "";
    }
    for (const std::string& c : spec.choices)  // string
        if (c == v) return v;
    return "";
}

bool ConfigurationDictionary::set(const ParamSpec& spec, const std::string& value, std::string* why) {
    const std::string c = canonical(spec, value);
    if (c.empty()) {
        m_values[spec.name] = canonical(spec, spec.defaultValue);
        if (why) *why = "parameter '" + spec.name + "': value '" + trim(value) + "' is not valid, default '" +
                        spec.defaultValue + "' used";
        return false;
    }
    m_values[spec.name] = c;
    return true;
}

const std::string& ConfigurationDictionary::get(const std::string& name) const {
    static const std::string empty;
    auto it = m_values.find(name);
    return it == m_values.end() ? empty : it->second;
}
double ConfigurationDictionary::getDouble(const std::string& name) const { return std::strtod(get(name).c_str(), nullptr); }
int64_t ConfigurationDictionary::getInt(const std::string& name) const { return std::strtoll(get(name).c_str(), nullptr, 10); }
bool ConfigurationDictionary::getBool(const std::string& name) const { return get(name) == "true"; }
DataType ConfigurationDictionary::getDataType(const std::string& name) const {
    DataType t = DataType::Float;
    parseDataType(get(name), t);
    return t;
}

// ---------------------------------------------------------------------------- records

std::shared_ptr<const Geometry> Geometry::copyOf(const sb_geometry& src) {
    auto g = std::make_shared<Geometry>();
    g->g = src;
    g->elementX.assign(src.element_x_mm, src.element_x_mm + src.num_elements);
    g->elementY.assign(src.element_y_mm, src.element_y_mm + src.num_elements);
    g->depths.assign(src.depths_mm, src.depths_mm + src.num_depths);
    g->scanlines.assign(src.scanlines, src.scanlines + src.num_rx);
    if (src.element_to_channel) g->elementToChannel.assign(src.element_to_channel, src.element_to_channel + src.num_elements);
    g->g.element_x_mm = g->elementX.data();
    g->g.element_y_mm = g->elementY.data();
    g->g.depths_mm = g->depths.data();
    g->g.scanlines = g->scanlines.data();
    g->g.element_to_channel = src.element_to_channel ? g->elementToChannel.data() : nullptr;
    return g;
}

std::shared_ptr<void> deviceBuffer(size_t bytes, sb_stream stream) {
    void* p = nullptr;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMallocAsync(&p, std::max<size_t>(bytes, 16), st) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return std::shared_ptr<void>(p, [st](void* q) { cudaFreeAsync(q, st); });
}

// ------------------------------------------------------------------------------ nodes

bool AbstractNode::setParameter(const std::string& name, const std::string& value) {
    std::lock_guard<std::mutex> l(m_mutex);
    const ParamSpec* spec = m_valueRangeDictionary.find(name);
    if (!spec) {
        m_lastError = "node " + m_nodeID + ": no parameter '" + name + "'";
        return false;
    }
    std::string why;
    const bool ok = m_configurationDictionary.set(*spec, value, &why);
    if (!ok) m_lastError = "node " + m_nodeID + ": " + why;
    configurationEntryChanged(name);
    return ok;
}

std::string AbstractNode::getParameter(const std::string& name) const {
    std::lock_guard<std::mutex> l(m_mutex);
    return m_configurationDictionary.get(name);
}

std::shared_ptr<RecordObject> AbstractNode::process(const std::shared_ptr<RecordObject>& in) {
    std::lock_guard<std::mutex> l(m_mutex);
    if (!in) return fail("no input");
    return processLocked(in);
}

std::string AbstractNode::lastError() const {
    std::lock_guard<std::mutex> l(m_mutex);
    return m_lastError;
}

void AbstractNode::finishConstruction() {
    for (const ParamSpec& s : m_valueRangeDictionary.all()) m_configurationDictionary.set(s, s.defaultValue, nullptr);
    configurationChanged();
}

std::shared_ptr<RecordObject> AbstractNode::fail(const std::string& why) {
    m_lastError = std::string(getType()) + " " + m_nodeID + ": " + why;
    return nullptr;
}

namespace {

const std::vector<std::string> kWindowNames = {"Rectangular", "Hann", "Hamming", "Gauss"};

int windowIndex(const std::string& name) {
    for (size_t i = 0; i < kWindowNames.size(); i++)
        if (kWindowNames[i] == name) return static_cast<int>(i);
    return 0;
}

std::string statusMessage(int st) { return "status " + std::to_string(st) + ": " + sb_last_error(); }

// Converts a float buffer into the requested output type with clampCast (in place when float).
std::shared_ptr<void> toOutputType(const std::shared_ptr<void>& f32, size_t n, DataType out, sb_stream stream,
                                   std::string* err) {
    if (out == DataType::Float) return f32;
    auto o = deviceBuffer(n * dtypeBytes(out), stream);
    if (!o) {
        *err = "device allocation failed";
        return nullptr;
    }
    const int st = sb_convert_run(f32.get(), SB_FLOAT32, o.get(), static_cast<int>(out), n, stream);
    if (st != SB_OK) {
        *err = statusMessage(st);
        return nullptr;
    }
    return o;
}

// Shared plan cache of the DAS nodes: rebuilt when the geometry object changes
// (BeamformingNode.cpp:141-150 compares the parameter pointer).
struct DasPlanCache {
    std::shared_ptr<const Geometry> geometry;
    sb_das_plan* plan = nullptr;
    ~DasPlanCache() { sb_das_plan_destroy(plan); }
    int get(const std::shared_ptr<const Geometry>& g, sb_das_plan** out) {
        if (plan && geometry == g) {
            *out = plan;
            return SB_OK;
        }
        sb_das_plan_destroy(plan);
        plan = nullptr;
        geometry = nullptr;
        const int st = sb_das_plan_create(&g->g, &plan);
        if (st != SB_OK) return st;
        geometry = g;
        *out = plan;
        return SB_OK;
    }
};

std::shared_ptr<ImageProperties> derivedProperties(const RecordObject& in, ImageProperties::State state) {
    auto p = in.properties ? std::make_shared<ImageProperties>(*in.properties) : std::make_shared<ImageProperties>();
    p->state = state;
    return p;
}

// ------------------------------------------------------------------- BeamformingNode
class BeamformingNode : public AbstractNode {
public:
    explicit BeamformingNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("fNumber", "double", 0.1, 4, "1", "F-Number");
        d.setChoices("windowType", "string", kWindowNames, "Rectangular", "RxWindow");
        d.setRange("windowParameter", "double", 0.0, 10.0, "0", "RxWindow parameter");
        d.setRange("speedOfSound", "double", 1000, 2000, "1540", "Speed of sound [m/s]");
        d.setChoices("beamformerType", "string", {"DelayAndSum", "DelayAndStdDev", "CoherenceFactorDelayAndSum", "TestSignal"},
                     "DelayAndSum", "RxBeamformer");
        d.setChoices("interpolateTransmits", "bool", {"false", "true"}, "false", "Interpolate Transmits");
        d.setRange("additionalOffset", "int32_t", -1000, 1000, "0", "Additional Offset [Samples]");
        d.setChoices("outputType", "DataType", {"float", "int16"}, "float", "Output type");
        finishConstruction();
    }
    const char* getType() const override { return "BeamformingNode"; }

protected:
    void configurationChanged() override {
        const auto& c = m_configurationDictionary;
        m_fNumber = c.getDouble("fNumber");
        m_windowType = windowIndex(c.get("windowType"));
        m_windowParameter = c.getDouble("windowParameter");
        m_speedOfSoundMMperS = c.getDouble("speedOfSound") * 1000.0;
        m_beamformerType = c.get("beamformerType");
        // BeamformingNode::updateImageProperties / configurationChanged (Beamformer/BeamformingNode.cpp:200-220)
        m_beamformer = m_beamformerType == "DelayAndStdDev"               ? SB_BF_DELAY_AND_STDDEV
                       : m_beamformerType == "CoherenceFactorDelayAndSum" ? SB_BF_COHERENCE_FACTOR_DAS
                       : m_beamformerType == "TestSignal"                 ? SB_BF_TEST_SIGNAL
                                                                          : SB_BF_DELAY_AND_SUM;
        m_interpolateTransmits = c.getBool("interpolateTransmits");
        m_additionalOffset = static_cast<int32_t>(c.getInt("additionalOffset"));
        m_outputType = c.getDataType("outputType");
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::RawData) return fail("input is not USRawData");
        auto raw = std::static_pointer_cast<USRawData>(in);
        if (raw->properties && raw->properties->state != ImageProperties::State::Raw)
            return fail("input is not raw channel data");
        if (raw->dtype != DataType::Int16 && raw->dtype != DataType::Float) return fail("input rawdata type not supported");
        sb_das_plan* plan = nullptr;
        int st = m_plans.get(raw->geometry, &plan);
        if (st != SB_OK) return fail(statusMessage(st));
        const sb_geometry& g = raw->geometry->g;
        auto out = deviceBuffer(static_cast<size_t>(g.num_depths) * g.num_rx * dtypeBytes(m_outputType), raw->stream);
        if (!out) return fail("device allocation failed");
        st = sb_das_run_beamformer(plan, m_beamformer, raw->data.get(), static_cast<int>(raw->dtype), out.get(),
                                   static_cast<int>(m_outputType), m_fNumber, m_speedOfSoundMMperS, m_windowType,
                                   static_cast<float>(m_windowParameter), m_interpolateTransmits ? 1 : 0,
                                   m_additionalOffset, raw->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        auto img = std::make_shared<USImage>();
        img->size[0] = g.num_rx;
        img->size[1] = g.num_depths;
        img->dtype = m_outputType;
        img->data = out;
        img->stream = raw->stream;
        auto p = derivedProperties(*raw, ImageProperties::State::RF);
        p->geometry = raw->geometry;
        p->numScanlines = g.num_rx;
        p->numSamples = g.num_depths;
        p->layoutX = g.rx_layout[0];
        p->layoutY = g.rx_layout[1];
        if (!(p->depthMM > 0)) p->depthMM = g.num_depths ? g.depths_mm[g.num_depths - 1] : 0.0;
        p->specific["Beamformer.FNumber"] = fmtDouble(m_fNumber);
        p->specific["Beamformer.WindowType"] = std::to_string(m_windowType);
        p->specific["Beamformer.WindowParameter"] = fmtDouble(m_windowParameter);
        p->specific["Beamformer.RxSpeedOfSound"] = fmtDouble(m_speedOfSoundMMperS);
        p->specific["Beamformer.BeamformerType"] = std::to_string(m_beamformer);  // the enum, streamed
        p->specific["Beamformer.InterpolateTransmits"] = m_interpolateTransmits ? "1" : "0";
        img->properties = p;
        return img;
    }

private:
    double m_fNumber = 1, m_windowParameter = 0, m_speedOfSoundMMperS = 1540e3;
    int m_windowType = 0;
    std::string m_beamformerType;
    int m_beamformer = SB_BF_DELAY_AND_SUM;
    bool m_interpolateTransmits = false;
    int32_t m_additionalOffset = 0;
    DataType m_outputType = DataType::Float;
    DasPlanCache m_plans;
};

// ---------------------------------------------------------------------- RawDelayNode
class RawDelayNode : public AbstractNode {
public:
    explicit RawDelayNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("fNumber", "double", 0.01, 4, "1", "F-Number");
        d.setChoices("windowType", "string", kWindowNames, "Rectangular", "RxWindow");
        d.setRange("windowParameter", "double", 0.0, 10.0, "0", "RxWindow parameter");
        d.setRange("speedOfSound", "double", 1000, 2000, "1540", "Speed of sound [m/s]");
        d.setChoices("outputType", "DataType", {"float", "int16"}, "float", "Output type");
        finishConstruction();
    }
    const char* getType() const override { return "RawDelayNode"; }

protected:
    void configurationChanged() override {
        const auto& c = m_configurationDictionary;
        m_fNumber = c.getDouble("fNumber");
        m_windowType = windowIndex(c.get("windowType"));
        m_windowParameter = c.getDouble("windowParameter");
        m_speedOfSoundMMperS = c.getDouble("speedOfSound") * 1000.0;
        m_outputType = c.getDataType("outputType");
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::RawData) return fail("input is not USRawData");
        auto raw = std::static_pointer_cast<USRawData>(in);
        if (raw->properties && raw->properties->state != ImageProperties::State::Raw)
            return fail("input is not raw channel data");
        if (raw->dtype != DataType::Int16 && raw->dtype != DataType::Float) return fail("input rawdata type not supported");
        sb_das_plan* plan = nullptr;
        int st = m_plans.get(raw->geometry, &plan);
        if (st != SB_OK) return fail(statusMessage(st));
        const sb_geometry& g = raw->geometry->g;
        const size_t n = static_cast<size_t>(g.num_rx) * g.num_channels * g.num_depths;
        auto out = deviceBuffer(n * dtypeBytes(m_outputType), raw->stream);
        if (!out) return fail("device allocation failed");
        st = sb_rawdelay_run(plan, raw->data.get(), static_cast<int>(raw->dtype), out.get(), static_cast<int>(m_outputType),
                             m_fNumber, m_speedOfSoundMMperS, m_windowType, static_cast<float>(m_windowParameter),
                             raw->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        auto r = std::make_shared<USRawData>();
        r->geometry = raw->geometry;
        r->data = out;
        r->dtype = m_outputType;
        r->numTx = g.num_rx;
        r->numChannels = g.num_channels;
        r->numSamples = g.num_depths;
        r->stream = raw->stream;
        auto p = derivedProperties(*raw, ImageProperties::State::RawDelayed);
        p->geometry = raw->geometry;
        p->numScanlines = g.num_rx;
        p->numSamples = g.num_depths;
        p->layoutX = g.rx_layout[0];
        p->layoutY = g.rx_layout[1];
        if (!(p->depthMM > 0)) p->depthMM = g.num_depths ? g.depths_mm[g.num_depths - 1] : 0.0;
        p->specific["Beamformer.FNumber"] = fmtDouble(m_fNumber);
        p->specific["Beamformer.RxSpeedOfSound"] = fmtDouble(m_speedOfSoundMMperS);
        r->properties = p;
        return r;
    }

private:
    double m_fNumber = 1, m_windowParameter = 0, m_speedOfSoundMMperS = 1540e3;
    int m_windowType = 0;
    DataType m_outputType = DataType::Float;
    DasPlanCache m_plans;
};

// ----------------------------------------------------------------- BeamformingMVNode
class BeamformingMVNode : public AbstractNode {
public:
    explicit BeamformingMVNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("subArraySize", "uint32_t", 0, 64, "0", "Sub-array size");
        d.setRange("temporalSmoothing", "uint32_t", 0, 10, "3", "temporal smoothing");
        d.setChoices("outputType", "DataType", {"float", "uint16"}, "float", "Output type");
        d.setRange("subArrayScalingPower", "double", 0.5, 3.0, "1.5", "Subarray count scaling power");
        d.setChoices("computeMeans", "bool", {"false", "true"}, "false", "compute signal means");
        // extensions (no reference counterpart): loading factor and the FP64 re-solve threshold
        d.setRange("diagonalLoadingScale", "double", 0.0, 100.0, "1", "Diagonal loading x trace/L (extension)");
        d.setRange("fp64Threshold", "double", 0.0, 1e30, "1000000", "FP64 re-solve above this condition estimate (extension)");
        finishConstruction();
    }
    const char* getType() const override { return "BeamformingMVNode"; }

protected:
    void configurationChanged() override {
        const auto& c = m_configurationDictionary;
        m_subArraySize = static_cast<uint32_t>(c.getInt("subArraySize"));
        m_temporalSmoothing = static_cast<uint32_t>(c.getInt("temporalSmoothing"));
        m_outputType = c.getDataType("outputType");
        m_scalingPower = c.getDouble("subArrayScalingPower");
        m_computeMeans = c.getBool("computeMeans");
        m_loading = c.getDouble("diagonalLoadingScale");
        m_fp64Threshold = c.getDouble("fp64Threshold");
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::RawData) return fail("input is not USRawData");
        auto raw = std::static_pointer_cast<USRawData>(in);
        if (!raw->properties || raw->properties->state != ImageProperties::State::RawDelayed)
            return fail("Cannot beamform undelayed RawData. Apply RawDelayNode first");
        if (raw->dtype != DataType::Int16 && raw->dtype != DataType::Float && raw->dtype != DataType::Complex64)
            return fail("input rawdata type is not supported");
        // the reference's output switch handles float and int16 only (BeamformingMVNode.cpp:96-114)
        if (m_outputType != DataType::Float) return fail("output image type not supported");
        const DataType outT = raw->dtype == DataType::Complex64 ? DataType::Complex64 : DataType::Float;
        const uint32_t nRx = raw->numTx, nCh = raw->numChannels, nS = raw->numSamples;
        auto out = deviceBuffer(static_cast<size_t>(nS) * nRx * dtypeBytes(outT), raw->stream);
        if (!out) return fail("device allocation failed");
        const int st = sb_mv_run(raw->data.get(), static_cast<int>(raw->dtype), out.get(), static_cast<int>(outT), nRx,
                                 nCh, nS, m_subArraySize, m_temporalSmoothing, m_scalingPower, m_computeMeans ? 1 : 0,
                                 static_cast<float>(m_loading), static_cast<float>(m_fp64Threshold), nullptr, raw->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        auto img = std::make_shared<USImage>();
        img->size[0] = nRx;
        img->size[1] = nS;
        img->dtype = outT;
        img->data = out;
        img->stream = raw->stream;
        auto p = derivedProperties(*raw, ImageProperties::State::RF);
        p->specific["BeamformingMVNode.subArraySize"] = std::to_string(m_subArraySize);
        p->specific["BeamformingMVNode.temporalSmoothing"] = std::to_string(m_temporalSmoothing);
        img->properties = p;
        return img;
    }

private:
    uint32_t m_subArraySize = 0, m_temporalSmoothing = 3;
    DataType m_outputType = DataType::Float;
    double m_scalingPower = 1.5, m_loading = 1.0, m_fp64Threshold = 1e6;
    bool m_computeMeans = false;
};

// ---------------------------------------------------------------- BeamformingMVpcgNode
// BeamformingMVpcgNode (Beamformer/BeamformingMVpcgNode.cpp:41-190): minimum variance on raw-delayed
// data with the weights from Jacobi-PCG; the convergence threshold is 10^convergenceThresholdExponent.
class BeamformingMVpcgNode : public AbstractNode {
public:
    explicit BeamformingMVpcgNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("subArraySize", "uint32_t", 0, 64, "0", "Sub-array size");
        d.setRange("temporalSmoothing", "uint32_t", 0, 10, "3", "temporal smoothing");
        d.setChoices("outputType", "DataType", {"float", "uint16"}, "float", "Output type");
        d.setRange("maxIterationsOverride", "uint32_t", 0, 10000, "0", "Max iterations override (if != 0)");
        d.setRange("convergenceThresholdExponent", "double", -100.0, 0.0, "-4", "Convergence threshold exponent");
        d.setRange("subArrayScalingPower", "double", 0.5, 3.0, "1.5", "Subarray count scaling power");
        d.setChoices("computeMeans", "bool", {"false", "true"}, "false", "compute signal means");
        finishConstruction();
    }
    const char* getType() const override { return "BeamformingMVpcgNode"; }

protected:
    void configurationChanged() override {
        const auto& c = m_configurationDictionary;
        m_subArraySize = static_cast<uint32_t>(c.getInt("subArraySize"));
        m_temporalSmoothing = static_cast<uint32_t>(c.getInt("temporalSmoothing"));
        m_outputType = c.getDataType("outputType");
        m_maxIterationsOverride = static_cast<uint32_t>(c.getInt("maxIterationsOverride"));
        m_convergenceThreshold = std::pow(10.0, c.getDouble("convergenceThresholdExponent"));
        m_scalingPower = c.getDouble("subArrayScalingPower");
        m_computeMeans = c.getBool("computeMeans");
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::RawData) return fail("input is not USRawData");
        auto raw = std::static_pointer_cast<USRawData>(in);
        if (!raw->properties || raw->properties->state != ImageProperties::State::RawDelayed)
            return fail("Cannot beamform undelayed RawData. Apply RawDelayNode first");
        if (raw->dtype != DataType::Int16 && raw->dtype != DataType::Float) return fail("input rawdata type is not supported");
        // the reference's output switch handles float and int16 only (BeamformingMVpcgNode.cpp:124-140)
        if (m_outputType != DataType::Float) return fail("output image type not supported");
        const uint32_t nRx = raw->numTx, nCh = raw->numChannels, nS = raw->numSamples;
        auto out = deviceBuffer(static_cast<size_t>(nS) * nRx * sizeof(float), raw->stream);
        if (!out) return fail("device allocation failed");
        const int st = sb_mv_pcg_run(raw->data.get(), static_cast<int>(raw->dtype), out.get(), SB_FLOAT32, nRx, nCh, nS,
                                     m_subArraySize, m_temporalSmoothing, m_maxIterationsOverride, m_convergenceThreshold,
                                     m_scalingPower, m_computeMeans ? 1 : 0, 1.0f, raw->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        auto img = std::make_shared<USImage>();
        img->size[0] = nRx;
        img->size[1] = nS;
        img->dtype = DataType::Float;
        img->data = out;
        img->stream = raw->stream;
        auto p = derivedProperties(*raw, ImageProperties::State::RF);
        p->specific["BeamformingMVNode.subArraySize"] = std::to_string(m_subArraySize);
        p->specific["BeamformingMVNode.temporalSmoothing"] = std::to_string(m_temporalSmoothing);
        img->properties = p;
        return img;
    }

private:
    uint32_t m_subArraySize = 0, m_temporalSmoothing = 3, m_maxIterationsOverride = 0;
    DataType m_outputType = DataType::Float;
    double m_convergenceThreshold = 1e-4, m_scalingPower = 1.5;
    bool m_computeMeans = false;
};

// ------------------------------------------------------------------ HilbertEnvelopeNode
// HilbertEnvelopeNode (Beamformer/HilbertEnvelopeNode.cpp:38-156): the analytic-signal envelope of each
// scanline over its whole length; "decimation" is kept as a parameter and property but, as in the
// reference (HilbertEnvelope::decimatedSignalLength), not applied.
class HilbertEnvelopeNode : public AbstractNode {
public:
    explicit HilbertEnvelopeNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("decimation", "uint32_t", 1, 100, "8", "Decimation");
        d.setChoices("outputType", "DataType", {"float", "int16"}, "float", "Output type");
        finishConstruction();
    }
    ~HilbertEnvelopeNode() override { sb_analytic_plan_destroy(m_plan); }
    const char* getType() const override { return "HilbertEnvelopeNode"; }

protected:
    void configurationChanged() override {
        m_decimation = static_cast<uint32_t>(m_configurationDictionary.getInt("decimation"));
        m_outputType = m_configurationDictionary.getDataType("outputType");
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::Image) return fail("input is not USImage");
        auto im = std::static_pointer_cast<USImage>(in);
        if (im->dtype != DataType::Int16 && im->dtype != DataType::Float) return fail("Input image type not supported.");
        const uint32_t nL = im->size[0], nS = im->size[1];
        if (!m_plan || m_planSamples != nS) {
            sb_analytic_plan_destroy(m_plan);
            m_plan = nullptr;
            const int st = sb_analytic_plan_create(nS, &m_plan);
            if (st != SB_OK) return fail(statusMessage(st));
            m_planSamples = nS;
        }
        auto out = deviceBuffer(static_cast<size_t>(nL) * nS * dtypeBytes(m_outputType), im->stream);
        if (!out) return fail("device allocation failed");
        const int st = sb_analytic_env_run(m_plan, im->data.get(), static_cast<int>(im->dtype), out.get(),
                                           static_cast<int>(m_outputType), nL, im->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        auto o = std::make_shared<USImage>();
        o->size[0] = nL;
        o->size[1] = nS;
        o->size[2] = 1;
        o->dtype = m_outputType;
        o->data = out;
        o->stream = im->stream;
        auto p = derivedProperties(*im, ImageProperties::State::EnvDetected);
        p->numSamples = nS;
        p->specific["Hilbert.Decimation"] = std::to_string(m_decimation);
        o->properties = p;
        return o;
    }

private:
    uint32_t m_decimation = 8, m_planSamples = 0;
    DataType m_outputType = DataType::Float;
    sb_analytic_plan* m_plan = nullptr;
};

// ------------------------------------------------------------ HilbertFirEnvelopeNode
class HilbertFirEnvelopeNode : public AbstractNode {
public:
    explicit HilbertFirEnvelopeNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("filterLength", "uint32_t", 1, 257, "65", "Filter Length");
        d.setChoices("outputType", "DataType", {"float", "int16"}, "float", "Output type");
        finishConstruction();
    }
    ~HilbertFirEnvelopeNode() override { sb_hilbert_plan_destroy(m_plan); }
    const char* getType() const override { return "HilbertFirEnvelopeNode"; }

protected:
    void configurationChanged() override {
        const uint32_t len = static_cast<uint32_t>(m_configurationDictionary.getInt("filterLength"));
        if (len != m_filterLength) {
            sb_hilbert_plan_destroy(m_plan);
            m_plan = nullptr;
            m_filterLength = len;
        }
        m_outputType = m_configurationDictionary.getDataType("outputType");
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::Image) return fail("input is not USImage");
        auto im = std::static_pointer_cast<USImage>(in);
        if (im->dtype != DataType::Float && im->dtype != DataType::Int16) return fail("input image type not supported");
        if (!m_plan) {
            const int st = sb_hilbert_plan_create(m_filterLength, &m_plan);
            if (st != SB_OK) return fail(statusMessage(st));
        }
        const size_t n = static_cast<size_t>(im->size[0]) * im->size[1];
        auto env = deviceBuffer(n * sizeof(float), im->stream);
        if (!env) return fail("device allocation failed");
        int st = sb_hilbert_env_run(m_plan, im->data.get(), static_cast<int>(im->dtype), env.get(), SB_FLOAT32, im->size[0],
                                    im->size[1], im->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        std::string err;
        auto out = toOutputType(env, n, m_outputType, im->stream, &err);
        if (!out) return fail(err);
        auto o = std::make_shared<USImage>();
        o->size[0] = im->size[0];
        o->size[1] = im->size[1];
        o->dtype = m_outputType;
        o->data = out;
        o->stream = im->stream;
        auto p = derivedProperties(*im, ImageProperties::State::EnvDetected);
        p->specific["HilbertFirEnvelope.FilterLength"] = std::to_string(m_filterLength);
        o->properties = p;
        return o;
    }

private:
    uint32_t m_filterLength = 0;
    DataType m_outputType = DataType::Float;
    sb_hilbert_plan* m_plan = nullptr;
};

// ------------------------------------------------------------------ IQDemodulatorNode
class IQDemodulatorNode : public AbstractNode {
public:
    explicit IQDemodulatorNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("decimation", "uint32_t", 1, 100, "8", "Decimation");
        d.setRange("referenceFrequency", "double", 1e6, 20e6, "7000000", "Reference frequency");
        for (int k = 0; k < 5; k++)
            d.setRange("referenceFrequencyAdd" + std::to_string(k), "double", 0, 20e6, "0",
                       "Reference frequency ADD" + std::to_string(k));
        d.setRange("weight", "double", 0, 5, "1", "Weight");
        for (int k = 0; k < 5; k++) d.setRange("weightAdd" + std::to_string(k), "double", 0, 5, "0", "Weight ADD" + std::to_string(k));
        d.setRange("bandwidth", "double", 0, 20e6, "1000000", "Bandwidth");
        for (int k = 0; k < 5; k++)
            d.setRange("bandwidthAdd" + std::to_string(k), "double", 0, 20e6, "1000000", "Bandwidth ADD" + std::to_string(k));
        d.setChoices("outputType", "DataType", {"float", "int16"}, "float", "Output type");
        finishConstruction();
    }
    ~IQDemodulatorNode() override { sb_iq_plan_destroy(m_plan); }
    const char* getType() const override { return "IQDemodulatorNode"; }

protected:
    void configurationChanged() override {
        const auto& c = m_configurationDictionary;
        m_decimation = static_cast<uint32_t>(c.getInt("decimation"));
        m_outputType = c.getDataType("outputType");
        // readFrequencyCompoundingSettings (IQDemodulatorNode.cpp:123-162): the list ends at the first
        // zero frequency or weight
        std::vector<double> f(6), w(6), b(6);
        f[0] = c.getDouble("referenceFrequency");
        w[0] = c.getDouble("weight");
        b[0] = c.getDouble("bandwidth");
        for (int k = 0; k < 5; k++) {
            f[k + 1] = c.getDouble("referenceFrequencyAdd" + std::to_string(k));
            w[k + 1] = c.getDouble("weightAdd" + std::to_string(k));
            b[k + 1] = c.getDouble("bandwidthAdd" + std::to_string(k));
        }
        size_t n = 6;
        for (size_t k = 0; k < 6; k++)
            if (f[k] == 0.0 || w[k] == 0.0) {
                n = k;
                break;
            }
        f.resize(n);
        w.resize(n);
        b.resize(n);
        if (f != m_freqs || w != m_weights || b != m_bandwidths) {
            sb_iq_plan_destroy(m_plan);
            m_plan = nullptr;
            m_freqs = f;
            m_weights = w;
            m_bandwidths = b;
        }
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::Image) return fail("input is not USImage");
        auto im = std::static_pointer_cast<USImage>(in);
        if (im->dtype != DataType::Float && im->dtype != DataType::Int16) return fail("input image type not supported");
        if (m_freqs.empty()) return fail("no demodulation frequency configured");
        if (!m_plan) {
            const int st = sb_iq_plan_create(kSamplingFrequency, kCutoffFrequency, kLowpassLength, kBandpassLength,
                                             static_cast<uint32_t>(m_freqs.size()), m_freqs.data(), m_bandwidths.data(),
                                             m_weights.data(), &m_plan);
            if (st != SB_OK) return fail(statusMessage(st));
        }
        const uint32_t nL = im->size[0], nS = im->size[1];
        const uint32_t nOut = m_decimation > 1 ? nS / m_decimation : nS;  // IQDemodulator.cu:204-212
        const size_t n = static_cast<size_t>(nOut) * nL;
        auto env = deviceBuffer(n * sizeof(float), im->stream);
        if (!env) return fail("device allocation failed");
        int st = sb_iq_magnitude_run(m_plan, im->data.get(), static_cast<int>(im->dtype), env.get(), SB_FLOAT32, nL, nS,
                                     m_decimation, im->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        std::string err;
        auto out = toOutputType(env, n, m_outputType, im->stream, &err);
        if (!out) return fail(err);
        auto o = std::make_shared<USImage>();
        o->size[0] = nL;
        o->size[1] = nOut;
        o->dtype = m_outputType;
        o->data = out;
        o->stream = im->stream;
        auto p = derivedProperties(*im, ImageProperties::State::EnvDetected);
        p->numSamples = nOut;
        p->specific["Iqdemod.Decimation"] = std::to_string(m_decimation);
        p->specific["Iqdemod.SamplingFrequency"] = fmtDouble(kSamplingFrequency);
        p->specific["Iqdemod.CutoffFrequency"] = fmtDouble(kCutoffFrequency);
        o->properties = p;
        return o;
    }

private:
    static constexpr double kSamplingFrequency = 40e6, kCutoffFrequency = 2.5e6;  // IQDemodulatorNode.cpp:26-27
    static constexpr uint32_t kLowpassLength = 51, kBandpassLength = 51;         // :28-29
    uint32_t m_decimation = 8;
    DataType m_outputType = DataType::Float;
    std::vector<double> m_freqs, m_weights, m_bandwidths;
    sb_iq_plan* m_plan = nullptr;
};

// ------------------------------------------------------------------ LogCompressorNode
class LogCompressorNode : public AbstractNode {
public:
    explicit LogCompressorNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("dynamicRange", "double", 1, 200, "80", "Dynamic Range");
        d.setRange("gain", "double", 0.01, 2, "1", "Gain");
        d.setRange("inMax", "double", 10, 50000, "1024", "Max Input");
        d.setChoices("outputType", "DataType", {"float", "uint8"}, "float", "Output type");
        finishConstruction();
    }
    const char* getType() const override { return "LogCompressorNode"; }

protected:
    void configurationChanged() override {
        const auto& c = m_configurationDictionary;
        m_dynamicRange = c.getDouble("dynamicRange");
        m_gain = c.getDouble("gain");
        m_inMax = c.getDouble("inMax");
        m_outputType = c.getDataType("outputType");
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::Image) return fail("input is not USImage");
        auto im = std::static_pointer_cast<USImage>(in);
        const size_t n = static_cast<size_t>(im->size[0]) * im->size[1] * std::max<uint32_t>(im->size[2], 1);
        auto out = deviceBuffer(n * dtypeBytes(m_outputType), im->stream);
        if (!out) return fail("device allocation failed");
        const int st = sb_logcompress_run(im->data.get(), static_cast<int>(im->dtype), out.get(),
                                          static_cast<int>(m_outputType), n, m_dynamicRange, m_gain, m_inMax, im->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        auto o = std::make_shared<USImage>();
        std::copy(im->size, im->size + 3, o->size);
        o->dtype = m_outputType;
        o->data = out;
        o->stream = im->stream;
        auto p = derivedProperties(*im, ImageProperties::State::LogCompressed);
        p->specific["LogCompressor.DynamicRange"] = fmtDouble(m_dynamicRange);
        p->specific["LogCompressor.Gain"] = fmtDouble(m_gain);
        p->specific["LogCompressor.InMax"] = fmtDouble(m_inMax);
        o->properties = p;
        return o;
    }

private:
    double m_dynamicRange = 80, m_gain = 1, m_inMax = 1024;
    DataType m_outputType = DataType::Float;
};

// ----------------------------------------------------------------- TemporalFilterNode
// TemporalFilterNode (Beamformer/TemporalFilterNode.cpp:36-168): keeps the last numImages images of one
// size and data type (a change of either empties the store) and outputs their mean, weights 1, oldest
// first. "outputType" offers float and uint16 as the reference's dictionary does; the reference's filter
// exists for int16 and float outputs only, so uint16 is refused ("Image output type not supported").
class TemporalFilterNode : public AbstractNode {
public:
    explicit TemporalFilterNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("numImages", "uint32_t", 1, 50, "3", "Number of Images");
        d.setChoices("outputType", "DataType", {"float", "uint16"}, "float", "Output type");
        finishConstruction();
    }
    const char* getType() const override { return "TemporalFilterNode"; }

protected:
    void configurationChanged() override {
        m_numImages = static_cast<uint32_t>(m_configurationDictionary.getInt("numImages"));
        m_outputType = m_configurationDictionary.getDataType("outputType");
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::Image) return fail("input is not USImage");
        auto im = std::static_pointer_cast<USImage>(in);
        if (im->dtype != DataType::Int16 && im->dtype != DataType::Float) return fail("Image input type not supported");
        if (!std::equal(im->size, im->size + 3, m_size) || im->dtype != m_dtype) {
            std::copy(im->size, im->size + 3, m_size);
            m_dtype = im->dtype;
            m_stored.clear();
        }
        m_stored.push_back(im->data);
        while (m_stored.size() > m_numImages) m_stored.pop_front();
        if (m_outputType != DataType::Float && m_outputType != DataType::Int16)
            return fail("Image output type not supported");
        const size_t n = static_cast<size_t>(im->size[0]) * im->size[1] * std::max<uint32_t>(im->size[2], 1);
        auto out = deviceBuffer(n * dtypeBytes(m_outputType), im->stream);
        if (!out) return fail("device allocation failed");
        std::vector<const void*> images;
        for (const auto& d : m_stored) images.push_back(d.get());
        const int st = sb_temporal_filter_run(images.data(), static_cast<uint32_t>(images.size()), nullptr,
                                              static_cast<int>(m_dtype), out.get(), static_cast<int>(m_outputType), n,
                                              im->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        auto o = std::make_shared<USImage>();
        std::copy(im->size, im->size + 3, o->size);
        o->dtype = m_outputType;
        o->data = out;
        o->stream = im->stream;
        auto p = derivedProperties(*im, im->properties ? im->properties->state : ImageProperties::State::RF);
        p->specific["TemporalFilter.NumImages"] = std::to_string(m_numImages);
        o->properties = p;
        return o;
    }

private:
    uint32_t m_numImages = 3;
    DataType m_outputType = DataType::Float;
    uint32_t m_size[3] = {0, 0, 0};
    DataType m_dtype = DataType::Float;
    std::deque<std::shared_ptr<void>> m_stored;  // the images' buffers, oldest first
};

// ------------------------------------------------------------------ ScanConverterNode
class ScanConverterNode : public AbstractNode {
public:
    explicit ScanConverterNode(const std::string& id) : AbstractNode(id) {
        auto& d = m_valueRangeDictionary;
        d.setRange("imageResolution", "double", 0.01, 5, "0.1", "Forced image resolution");
        d.setChoices("imageResolutionForced", "bool", {"true", "false"}, "false", "Force image resolution");
        d.setChoices("outputType", "DataType", {"float", "int16", "uint8"}, "float", "Output type");
        finishConstruction();
    }
    ~ScanConverterNode() override { sb_scan_plan_destroy(m_plan); }
    const char* getType() const override { return "ScanConverterNode"; }

protected:
    void configurationChanged() override {
        const auto& c = m_configurationDictionary;
        m_imageResolution = c.getDouble("imageResolution");
        m_forceResolution = c.getBool("imageResolutionForced");
        m_outputType = c.getDataType("outputType");
    }
    std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) override {
        if (in->getType() != RecordType::Image) return fail("input is not USImage");
        auto im = std::static_pointer_cast<USImage>(in);
        const ImageProperties* pr = im->properties.get();
        if (!pr || !pr->geometry) return fail("image has no scanline geometry");
        if (im->dtype != DataType::Float && im->dtype != DataType::Int16 && im->dtype != DataType::Uint8)
            return fail("input image type not supported");
        const double res = m_forceResolution ? m_imageResolution : pr->imageResolutionMM;
        // rebuild the tables when the geometry, layout, depth, samples or resolution change
        // (ScanConverterNode.cpp:130-166)
        if (!m_plan || m_geometry != pr->geometry || m_numSamples != im->size[1] || m_depth != pr->depthMM || m_res != res) {
            sb_scan_plan_destroy(m_plan);
            m_plan = nullptr;
            const int st = sb_scan_plan_create(pr->geometry->g.scanlines, pr->layoutX, pr->layoutY, im->size[1], pr->depthMM,
                                               res, &m_plan);
            if (st != SB_OK) return fail(statusMessage(st));
            m_geometry = pr->geometry;
            m_numSamples = im->size[1];
            m_depth = pr->depthMM;
            m_res = res;
        }
        uint32_t sz[3];
        int st = sb_scan_image_size(m_plan, sz);
        if (st != SB_OK) return fail(statusMessage(st));
        const size_t n = static_cast<size_t>(sz[0]) * sz[1] * sz[2];
        auto out = deviceBuffer(n * dtypeBytes(m_outputType), im->stream);
        if (!out) return fail("device allocation failed");
        st = sb_scan_run(m_plan, im->data.get(), static_cast<int>(im->dtype), out.get(), static_cast<int>(m_outputType),
                         im->stream);
        if (st != SB_OK) return fail(statusMessage(st));
        auto o = std::make_shared<USImage>();
        std::copy(sz, sz + 3, o->size);
        o->dtype = m_outputType;
        o->data = out;
        o->stream = im->stream;
        auto p = derivedProperties(*im, ImageProperties::State::ScanConverted);
        p->imageResolutionMM = res;
        o->properties = p;
        return o;
    }

private:
    double m_imageResolution = 0.1;
    bool m_forceResolution = false;
    DataType m_outputType = DataType::Float;
    sb_scan_plan* m_plan = nullptr;
    std::shared_ptr<const Geometry> m_geometry;
    uint32_t m_numSamples = 0;
    double m_depth = -1, m_res = -1;
};

using Creator = std::function<std::unique_ptr<AbstractNode>(const std::string&)>;
const std::vector<std::pair<std::string, Creator>>& creators() {
    static const std::vector<std::pair<std::string, Creator>> c = {
        {"BeamformingNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new BeamformingNode(id)); }},
        {"RawDelayNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new RawDelayNode(id)); }},
        {"BeamformingMVNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new BeamformingMVNode(id)); }},
        {"BeamformingMVpcgNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new BeamformingMVpcgNode(id)); }},
        {"HilbertFirEnvelopeNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new HilbertFirEnvelopeNode(id)); }},
        {"HilbertEnvelopeNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new HilbertEnvelopeNode(id)); }},
        {"IQDemodulatorNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new IQDemodulatorNode(id)); }},
        {"LogCompressorNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new LogCompressorNode(id)); }},
        {"ScanConverterNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new ScanConverterNode(id)); }},
        {"TemporalFilterNode", [](const std::string& id) { return std::unique_ptr<AbstractNode>(new TemporalFilterNode(id)); }},
    };
    return c;
}

// ------------------------------------------------------------------------ XML reader
// Elements, attributes, text, comments and the declaration; enough for SUPRA's config files.
struct XmlNode {
    std::string name;
    std::map<std::string, std::string> attrs;
    std::string text;
    std::vector<std::unique_ptr<XmlNode>> children;
    std::vector<const XmlNode*> all(const std::string& n) const {
        std::vector<const XmlNode*> r;
        for (const auto& c : children)
            if (c->name == n) r.push_back(c.get());
        return r;
    }
    const XmlNode* first(const std::string& n) const {
        for (const auto& c : children)
            if (c->name == n) return c.get();
        return nullptr;
    }
};

class XmlParser {
public:
    explicit XmlParser(const std::string& s) : m_s(s) {}
    std::unique_ptr<XmlNode> parse(std::string* err) {
        skipMisc();
        auto root = element(err);
        return root;
    }

private:
    const std::string& m_s;
    size_t m_i = 0;
    bool starts(const char* p) const { return m_s.compare(m_i, std::strlen(p), p) == 0; }
    void skipWs() {
        while (m_i < m_s.size() && std::isspace(static_cast<unsigned char>(m_s[m_i]))) m_i++;
    }
    void skipMisc() {
        for (;;) {
            skipWs();
            if (starts("<?")) {
                const size_t e = m_s.find("?>", m_i);
                m_i = e == std::string::npos ? m_s.size() : e + 2;
            } else if (starts("<!--")) {
                const size_t e = m_s.find("-->", m_i);
                m_i = e == std::string::npos ? m_s.size() : e + 3;
            } else {
                return;
            }
        }
    }
    std::string nameToken() {
        const size_t a = m_i;
        while (m_i < m_s.size() && (std::isalnum(static_cast<unsigned char>(m_s[m_i])) || m_s[m_i] == '_' || m_s[m_i] == '-' ||
                                    m_s[m_i] == ':' || m_s[m_i] == '.'))
            m_i++;
        return m_s.substr(a, m_i - a);
    }
    static std::string unescape(const std::string& t) {
        std::string r;
        for (size_t i = 0; i < t.size(); i++) {
            if (t[i] == '&') {
                const size_t e = t.find(';', i);
                if (e != std::string::npos) {
                    const std::string ent = t.substr(i + 1, e - i - 1);
                    if (ent == "lt") r += '<';
                    else if (ent == "gt") r += '>';
                    else if (ent == "amp") r += '&';
                    else if (ent == "quot") r += '"';
                    else if (ent == "apos") r += '\'';
                    else r += t.substr(i, e - i + 1);
                    i = e;
                    continue;
                }
            }
            r += t[i];
        }
        return r;
    }
    std::unique_ptr<XmlNode> element(std::string* err) {
        if (!starts("<")) {
            *err = "xml: element expected at offset " + std::to_string(m_i);
            return nullptr;
        }
        m_i++;
        auto n = std::make_unique<XmlNode>();
        n->name = nameToken();
        if (n->name.empty()) {
            *err = "xml: element name expected at offset " + std::to_string(m_i);
            return nullptr;
        }
        for (;;) {
            skipWs();
            if (starts("/>")) {
                m_i += 2;
                return n;
            }
            if (starts(">")) {
                m_i++;
                break;
            }
            const std::string an = nameToken();
            skipWs();
            if (an.empty() || !starts("=")) {
                *err = "xml: attribute expected in <" + n->name + ">";
                return nullptr;
            }
            m_i++;
            skipWs();
            const char q = m_i < m_s.size() ? m_s[m_i] : '\0';
            if (q != '"' && q != '\'') {
                *err = "xml: quoted attribute value expected in <" + n->name + ">";
                return nullptr;
            }
            const size_t e = m_s.find(q, m_i + 1);
            if (e == std::string::npos) {
                *err = "xml: unterminated attribute in <" + n->name + ">";
                return nullptr;
            }
            n->attrs[an] = unescape(m_s.substr(m_i + 1, e - m_i - 1));
            m_i = e + 1;
        }
        for (;;) {
            if (m_i >= m_s.size()) {
                *err = "xml: <" + n->name + "> not closed";
                return nullptr;
            }
            if (starts("<!--")) {
                const size_t e = m_s.find("-->", m_i);
                m_i = e == std::string::npos ? m_s.size() : e + 3;
            } else if (starts("</")) {
                m_i += 2;
                const std::string cn = nameToken();
                skipWs();
                if (cn != n->name || !starts(">")) {
                    *err = "xml: </" + cn + "> does not close <" + n->name + ">";
                    return nullptr;
                }
                m_i++;
                return n;
            } else if (starts("<")) {
                auto c = element(err);
                if (!c) return nullptr;
                n->children.push_back(std::move(c));
            } else {
                const size_t e = m_s.find('<', m_i);
                n->text += unescape(m_s.substr(m_i, (e == std::string::npos ? m_s.size() : e) - m_i));
                m_i = e == std::string::npos ? m_s.size() : e;
            }
        }
    }
};

}  // namespace

std::unique_ptr<AbstractNode> createNode(const std::string& type, const std::string& nodeID) {
    for (const auto& c : creators())
        if (c.first == type) return c.second(nodeID);
    return nullptr;
}

std::vector<std::string> nodeTypes() {
    std::vector<std::string> r;
    for (const auto& c : creators()) r.push_back(c.first);
    return r;
}

AbstractNode* Graph::node(const std::string& id) const {
    auto it = m_nodes.find(id);
    return it == m_nodes.end() ? nullptr : it->second.get();
}

std::unique_ptr<Graph> Graph::fromXml(const std::string& xml, std::string* error) {
    std::string err;
    auto root = XmlParser(xml).parse(&err);
    if (!root) {
        if (error) *error = err;
        return nullptr;
    }
    if (root->name != "supra_config") {
        if (error) *error = "xml: root element is <" + root->name + ">, expected <supra_config>";
        return nullptr;
    }
    std::unique_ptr<Graph> g(new Graph());
    std::vector<std::string> inputs;
    const XmlNode* devices = root->first("devices");
    if (devices) {
        if (const XmlNode* ins = devices->first("inputs"))
            for (const XmlNode* i : ins->all("input")) {
                inputs.push_back(i->attrs.count("id") ? i->attrs.at("id") : "");
                if (inputs.size() == 1) {  // the first input's type and parameters (a recorded-data input is replayed)
                    g->m_inputType = i->attrs.count("type") ? i->attrs.at("type") : "";
                    for (const XmlNode* p : i->all("param"))
                        if (p->attrs.count("name")) g->m_inputParams[p->attrs.at("name")] = trim(p->text);
                }
            }
        if (const XmlNode* nodes = devices->first("nodes")) {
            for (const XmlNode* n : nodes->all("node")) {
                const std::string type = n->attrs.count("type") ? n->attrs.at("type") : "";
                const std::string id = n->attrs.count("id") ? n->attrs.at("id") : "";
                auto node = createNode(type, id);
                if (!node) {
                    g->m_skipped.push_back(id);  // outside the receive path: passed through
                    continue;
                }
                for (const XmlNode* p : n->all("param")) {
                    const std::string name = p->attrs.count("name") ? p->attrs.at("name") : "";
                    if (!node->getValueRangeDictionary().find(name)) continue;  // the reference ignores unknown keys
                    node->setParameter(name, trim(p->text));
                }
                g->m_nodes[id] = std::move(node);
            }
        }
    }
    // connections: follow the first outgoing edge from the (first) input through the nodes
    std::multimap<std::string, std::string> edges;
    if (const XmlNode* cons = root->first("connections"))
        for (const XmlNode* c : cons->all("connection")) {
            const XmlNode* f = c->first("from");
            const XmlNode* t = c->first("to");
            if (f && t && f->attrs.count("id") && t->attrs.count("id")) edges.emplace(f->attrs.at("id"), t->attrs.at("id"));
        }
    std::string cur;
    if (!inputs.empty()) cur = inputs.front();
    else if (!edges.empty()) cur = edges.begin()->first;
    std::vector<std::string> seen;
    for (;;) {
        auto it = edges.find(cur);
        if (it == edges.end()) break;
        cur = it->second;
        if (std::find(seen.begin(), seen.end(), cur) != seen.end()) break;  // cycle
        seen.push_back(cur);
        if (g->m_nodes.count(cur)) g->m_chain.push_back(cur);
    }
    if (g->m_chain.empty()) {
        for (const auto& kv : g->m_nodes) g->m_chain.push_back(kv.first);  // no connections: declaration order lost, id order
    }
    return g;
}

std::shared_ptr<RecordObject> Graph::process(const std::shared_ptr<RecordObject>& in, std::string* error) {
    std::shared_ptr<RecordObject> cur = in;
    for (const std::string& id : m_chain) {
        AbstractNode* n = node(id);
        cur = n->process(cur);
        if (!cur) {
            if (error) *error = n->lastError();
            return nullptr;
        }
    }
    return cur;
}

}  // namespace supra_b200

// ------------------------------------------------------------------------- C entry points

using namespace supra_b200;

struct sb_node {
    std::unique_ptr<AbstractNode> node;
    std::shared_ptr<RecordObject> last;      // keeps the last output alive until the next call
    std::shared_ptr<const Geometry> geometry;  // reused while the caller's geometry is unchanged
};

struct sb_graph {
    std::unique_ptr<Graph> graph;
    std::shared_ptr<RecordObject> last;
    std::shared_ptr<const Geometry> geometry;
    // replay of a recorded-data input (UltrasoundInterfaceRawDataMock)
    sb_mock_meta* meta = nullptr;
    sb_mock_reader* reader = nullptr;
    void* frame = nullptr;  // device frame buffer, reused frame after frame on the caller's stream
    ~sb_graph() {
        last.reset();
        sb_mock_reader_destroy(reader);
        sb_mock_meta_destroy(meta);
        if (frame) cudaFree(frame);  // cudaFree waits for the work that may still read it
    }
};

namespace {

int nodeFail(const std::string& msg, int code = SB_ERR_INVALID_ARG) {
    sb::setError("%s", msg.c_str());
    return code;
}

template <typename T> bool sameArray(const std::vector<T>& a, const T* b, size_t n) {
    if (a.size() != n || (n && !b)) return false;
    return n == 0 || std::memcmp(a.data(), b, n * sizeof(T)) == 0;
}

// The cached copy when its content equals `g` (the geometry object's identity then stays the same,
// so the node keeps its plans), otherwise a new copy.
std::shared_ptr<const Geometry> geometryFor(std::shared_ptr<const Geometry>& cache, const sb_geometry& g) {
    if (cache) {
        const sb_geometry& c = cache->g;
        const bool same = c.num_elements == g.num_elements && c.element_layout[0] == g.element_layout[0] &&
                          c.element_layout[1] == g.element_layout[1] && c.num_channels == g.num_channels &&
                          c.num_samples == g.num_samples && c.num_tx == g.num_tx && c.num_rx == g.num_rx &&
                          c.rx_layout[0] == g.rx_layout[0] && c.rx_layout[1] == g.rx_layout[1] &&
                          c.num_depths == g.num_depths && c.sampling_frequency_hz == g.sampling_frequency_hz &&
                          sameArray(cache->elementX, g.element_x_mm, g.num_elements) &&
                          sameArray(cache->elementY, g.element_y_mm, g.num_elements) &&
                          sameArray(cache->depths, g.depths_mm, g.num_depths) &&
                          sameArray(cache->scanlines, g.scanlines, g.num_rx) &&
                          (g.element_to_channel ? sameArray(cache->elementToChannel, g.element_to_channel, g.num_elements)
                                                : cache->elementToChannel.empty());
        if (same) return cache;
    }
    cache = Geometry::copyOf(g);
    return cache;
}

std::shared_ptr<RecordObject> recordFromRaw(std::shared_ptr<const Geometry>& cache, const sb_geometry* geometry,
                                            const void* data, int dtype, int delayed, uint32_t num_tx,
                                            uint32_t num_channels, uint32_t num_samples, double depth_mm,
                                            double image_resolution_mm, sb_stream stream) {
    auto r = std::make_shared<USRawData>();
    r->geometry = geometryFor(cache, *geometry);
    r->data = std::shared_ptr<void>(const_cast<void*>(data), [](void*) {});  // caller-owned
    r->dtype = static_cast<DataType>(dtype);
    r->numTx = num_tx;
    r->numChannels = num_channels;
    r->numSamples = num_samples;
    r->stream = stream;
    auto p = std::make_shared<ImageProperties>();
    p->state = delayed ? ImageProperties::State::RawDelayed : ImageProperties::State::Raw;
    p->geometry = r->geometry;
    p->imageResolutionMM = image_resolution_mm > 0 ? image_resolution_mm : 0.1;
    p->depthMM = depth_mm > 0 ? depth_mm : (geometry->num_depths ? geometry->depths_mm[geometry->num_depths - 1] : 0.0);
    p->layoutX = geometry->rx_layout[0];
    p->layoutY = geometry->rx_layout[1];
    r->properties = p;
    return r;
}

// A caller-owned device image as a USImage record (state as in sb_record; geometry optional).
std::shared_ptr<RecordObject> recordFromImage(std::shared_ptr<const Geometry>& cache, const sb_geometry* geometry,
                                              const void* data, int dtype, int state, const uint32_t size[3],
                                              double depth_mm, double image_resolution_mm, sb_stream stream) {
    auto im = std::make_shared<USImage>();
    im->data = std::shared_ptr<void>(const_cast<void*>(data), [](void*) {});  // caller-owned
    im->dtype = static_cast<DataType>(dtype);
    std::copy(size, size + 3, im->size);
    if (im->size[2] == 0) im->size[2] = 1;
    im->stream = stream;
    auto p = std::make_shared<ImageProperties>();
    p->state = static_cast<ImageProperties::State>(state);
    if (geometry) {
        p->geometry = geometryFor(cache, *geometry);
        p->layoutX = geometry->rx_layout[0];
        p->layoutY = geometry->rx_layout[1];
        if (!(depth_mm > 0) && geometry->num_depths) depth_mm = geometry->depths_mm[geometry->num_depths - 1];
    }
    p->numScanlines = size[0];
    p->numSamples = size[1];
    p->depthMM = depth_mm > 0 ? depth_mm : 0.0;
    p->imageResolutionMM = image_resolution_mm > 0 ? image_resolution_mm : 0.1;
    im->properties = p;
    return im;
}

void describe(const std::shared_ptr<RecordObject>& rec, sb_record* out) {
    std::memset(out, 0, sizeof(*out));
    if (!rec) return;
    if (rec->getType() == RecordType::Image) {
        auto im = std::static_pointer_cast<USImage>(rec);
        out->is_image = 1;
        out->data = im->data.get();
        out->dtype = static_cast<int>(im->dtype);
        out->size[0] = im->size[0];
        out->size[1] = im->size[1];
        out->size[2] = im->size[2];
    } else {
        auto r = std::static_pointer_cast<USRawData>(rec);
        out->is_image = 0;
        out->data = r->data.get();
        out->dtype = static_cast<int>(r->dtype);
        out->size[0] = r->numSamples;
        out->size[1] = r->numChannels;
        out->size[2] = r->numTx;
    }
    out->state = rec->properties ? static_cast<int>(rec->properties->state) : 0;
}

void copyString(const std::string& s, char* buf, size_t len) {
    if (!buf || len == 0) return;
    const size_t n = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
}

}  // namespace

extern "C" {

int sb_node_create(const char* type, const char* node_id, sb_node** out) {
    if (!type || !node_id || !out) return nodeFail("sb_node_create: null argument");
    *out = nullptr;
    auto n = createNode(type, node_id);
    if (!n) return nodeFail(std::string("sb_node_create: unknown node type ") + type);
    *out = new sb_node{std::move(n), nullptr};
    return SB_OK;
}

int sb_node_destroy(sb_node* node) {
    delete node;
    return SB_OK;
}

int sb_node_set_param(sb_node* node, const char* name, const char* value) {
    if (!node || !name || !value) return nodeFail("sb_node_set_param: null argument");
    if (!node->node->setParameter(name, value)) return nodeFail(node->node->lastError());
    return SB_OK;
}

int sb_node_get_param(const sb_node* node, const char* name, char* value, size_t value_len) {
    if (!node || !name) return nodeFail("sb_node_get_param: null argument");
    if (!node->node->getValueRangeDictionary().find(name)) return nodeFail(std::string("sb_node_get_param: no parameter ") + name);
    copyString(node->node->getParameter(name), value, value_len);
    return SB_OK;
}

int sb_node_param_count(const sb_node* node) {
    if (!node) return nodeFail("sb_node_param_count: null node");
    return static_cast<int>(node->node->getValueRangeDictionary().all().size());
}

int sb_node_param_info(const sb_node* node, int index, char* name, char* type, char* range, char* default_value,
                       size_t len) {
    if (!node) return nodeFail("sb_node_param_info: null node");
    const auto& all = node->node->getValueRangeDictionary().all();
    if (index < 0 || index >= static_cast<int>(all.size())) return nodeFail("sb_node_param_info: index out of range");
    const ParamSpec& s = all[index];
    copyString(s.name, name, len);
    copyString(s.type, type, len);
    std::string r;
    if (s.isRange) r = fmtDouble(s.min) + ".." + fmtDouble(s.max);
    else
        for (size_t i = 0; i < s.choices.size(); i++) r += (i ? "|" : "") + s.choices[i];
    copyString(r, range, len);
    copyString(s.defaultValue, default_value, len);
    return SB_OK;
}

int sb_node_type_count(void) { return static_cast<int>(nodeTypes().size()); }

int sb_node_type_name(int index, char* name, size_t len) {
    const auto t = nodeTypes();
    if (index < 0 || index >= static_cast<int>(t.size())) return nodeFail("sb_node_type_name: index out of range");
    copyString(t[index], name, len);
    return SB_OK;
}

int sb_node_process_raw(sb_node* node, const sb_geometry* geometry, const void* data, int dtype, int delayed,
                        uint32_t num_tx, uint32_t num_channels, uint32_t num_samples, double depth_mm,
                        double image_resolution_mm, sb_stream stream, sb_record* out) {
    if (!node || !geometry || !data || !out) return nodeFail("sb_node_process_raw: null argument");
    auto rec = recordFromRaw(node->geometry, geometry, data, dtype, delayed, num_tx, num_channels, num_samples,
                             depth_mm, image_resolution_mm, stream);
    node->last = node->node->process(rec);
    if (!node->last) return nodeFail(node->node->lastError(), SB_ERR_UNSUPPORTED);
    describe(node->last, out);
    return SB_OK;
}

int sb_node_process_image(sb_node* node, const sb_geometry* geometry, const void* data, int dtype, int state,
                          const uint32_t size[3], double depth_mm, double image_resolution_mm, sb_stream stream,
                          sb_record* out) {
    if (!node || !data || !size || !out) return nodeFail("sb_node_process_image: null argument");
    if (state < 0 || state > 5) return nodeFail("sb_node_process_image: state not in [0, 5]", SB_ERR_INVALID_ARG);
    auto rec = recordFromImage(node->geometry, geometry, data, dtype, state, size, depth_mm, image_resolution_mm, stream);
    node->last = node->node->process(rec);
    if (!node->last) return nodeFail(node->node->lastError(), SB_ERR_UNSUPPORTED);
    describe(node->last, out);
    return SB_OK;
}

int sb_node_process_last(sb_node* node, sb_node* upstream, sb_record* out) {
    if (!node || !upstream || !out) return nodeFail("sb_node_process_last: null argument");
    if (!upstream->last) return nodeFail("sb_node_process_last: the upstream node has no output");
    node->last = node->node->process(upstream->last);
    if (!node->last) return nodeFail(node->node->lastError(), SB_ERR_UNSUPPORTED);
    describe(node->last, out);
    return SB_OK;
}

int sb_graph_create_xml(const char* xml_text, sb_graph** out) {
    if (!xml_text || !out) return nodeFail("sb_graph_create_xml: null argument");
    *out = nullptr;
    std::string err;
    auto g = Graph::fromXml(xml_text, &err);
    if (!g) return nodeFail("sb_graph_create_xml: " + err);
    *out = new sb_graph{std::move(g), nullptr};
    return SB_OK;
}

int sb_graph_destroy(sb_graph* graph) {
    delete graph;
    return SB_OK;
}

int sb_graph_chain(const sb_graph* graph, char* ids, size_t len) {
    if (!graph) return nodeFail("sb_graph_chain: null graph");
    std::string s;
    for (size_t i = 0; i < graph->graph->chain().size(); i++) s += (i ? "," : "") + graph->graph->chain()[i];
    copyString(s, ids, len);
    return static_cast<int>(graph->graph->chain().size());
}

int sb_graph_node_get_param(const sb_graph* graph, const char* node_id, const char* name, char* value, size_t len) {
    if (!graph || !node_id || !name) return nodeFail("sb_graph_node_get_param: null argument");
    AbstractNode* n = graph->graph->node(node_id);
    if (!n) return nodeFail(std::string("sb_graph_node_get_param: no node ") + node_id);
    if (!n->getValueRangeDictionary().find(name)) return nodeFail(std::string("sb_graph_node_get_param: no parameter ") + name);
    copyString(n->getParameter(name), value, len);
    return SB_OK;
}

int sb_graph_process_raw(sb_graph* graph, const sb_geometry* geometry, const void* data, int dtype, uint32_t num_tx,
                         uint32_t num_channels, uint32_t num_samples, double depth_mm, double image_resolution_mm,
                         sb_stream stream, sb_record* out) {
    if (!graph || !geometry || !data || !out) return nodeFail("sb_graph_process_raw: null argument");
    auto rec = recordFromRaw(graph->geometry, geometry, data, dtype, 0, num_tx, num_channels, num_samples, depth_mm,
                             image_resolution_mm, stream);
    std::string err;
    graph->last = graph->graph->process(rec, &err);
    if (!graph->last) return nodeFail("sb_graph_process_raw: " + err, SB_ERR_UNSUPPORTED);
    describe(graph->last, out);
    return SB_OK;
}

int sb_graph_process_next(sb_graph* graph, double image_resolution_mm, sb_stream stream, int* last_frame,
                          sb_record* out) {
    if (!graph || !out) return nodeFail("sb_graph_process_next: null argument");
    if (last_frame) *last_frame = 0;
    Graph& G = *graph->graph;
    if (G.inputType() != "UltrasoundInterfaceRawDataMock")
        return nodeFail("sb_graph_process_next: the configuration's input is " +
                        (G.inputType().empty() ? std::string("missing") : G.inputType()) +
                        ", not UltrasoundInterfaceRawDataMock");
    if (!graph->reader) {
        // UltrasoundInterfaceRawDataMock::initializeDevice (SupraLib/InputOutput/UltrasoundInterfaceRawDataMock.cpp:47-92)
        auto flag = [&](const char* k) {
            const std::string v = G.inputParam(k);
            return v == "1" || v == "true";
        };
        int st = sb_mock_meta_read(G.inputParam("mockMetaDataFilename").c_str(), &graph->meta);
        if (st != SB_OK) return st;
        st = sb_mock_reader_create(graph->meta, G.inputParam("mockDataFilename").c_str(), flag("singleImage") ? 1 : 0,
                                   flag("streamSequenceOnce") ? 1 : 0, &graph->reader);
        if (st != SB_OK) return st;
        uint64_t bytes = 0;
        sb_mock_reader_info(graph->reader, &bytes, nullptr, nullptr);
        const cudaError_t e = cudaMalloc(&graph->frame, bytes);
        if (e != cudaSuccess) {
            graph->frame = nullptr;
            return nodeFail(std::string("sb_graph_process_next: frame buffer: ") + cudaGetErrorString(e), SB_ERR_NO_MEMORY);
        }
    }
    int last = 0;
    int st = sb_mock_reader_next(graph->reader, graph->frame, stream, &last);
    if (st != SB_OK) return st;
    sb_geometry g;
    double depth = 0.0, c = 0.0;
    sb_mock_meta_geometry(graph->meta, &g, &depth, &c);
    auto rec = recordFromRaw(graph->geometry, &g, graph->frame, SB_INT16, 0, g.num_tx, g.num_channels, g.num_samples,
                             depth, image_resolution_mm, stream);
    std::string err;
    graph->last = G.process(rec, &err);
    if (!graph->last) return nodeFail("sb_graph_process_next: " + err, SB_ERR_UNSUPPORTED);
    describe(graph->last, out);
    if (last_frame) *last_frame = last;
    return SB_OK;
}

}  // extern "C"
