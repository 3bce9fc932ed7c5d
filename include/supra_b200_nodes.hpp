/* supra_b200 node layer (C++): the processing nodes of SUPRA's receive path re-hosted on the C ABI.
 *
 * Mirrors the reference's node interface (SupraLib/AbstractNode.h:41-121): a node has an ID, a
 * value-range dictionary with the reference's parameter names, types, ranges and defaults, a
 * configuration dictionary validated against it (invalid entries fall back to the default, as
 * ConfigurationDictionary::checkEntriesAndLog does), configurationChanged /
 * configurationEntryChanged under the node mutex, and one processing function that takes and
 * returns a RecordObject (the body of the reference's tbb function_node). Type or state mismatches
 * return nullptr with the reason in lastError(), as the reference logs and returns nullptr.
 *
 * Records mirror USRawData (Beamformer/USRawData.h:24-80) and USImage (SupraLib/USImage.h:28): device
 * buffers in the reference layouts, the stream they are ordered on, and the image properties the
 * downstream nodes read (state, geometry, sizes, depth, resolution, specific parameters). Outputs
 * are allocated stream-ordered on the input's stream and freed the same way when the last
 * reference is dropped. Nothing synchronises the host (MV reads its statistics only on request).
 *
 * The graph runner builds nodes and connections from the reference's XML configuration format
 * (<supra_config><devices><nodes><node type id><param name type>value</param>... and
 * <connections><connection><from id port/><to id port/>) and pushes a record through the chain in
 * connection order, single-threaded (the reference's TBB flow graph is not rebuilt).
 */
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "supra_b200.h"

namespace supra_b200 {

enum class DataType { Int16 = SB_INT16, Float = SB_FLOAT32, Uint8 = SB_UINT8, Complex64 = SB_COMPLEX64, Uint16 = SB_UINT16 };
const char* dataTypeName(DataType t);
bool parseDataType(const std::string& s, DataType& t);  // SUPRA's names: int16, int16_t, float, uint8, uint8_t, ...

// One parameter of a node, as m_valueRangeDictionary.set<T>(name, ...) declares it.
struct ParamSpec {
    std::string name, type, label, defaultValue;  // type: double, uint32_t, int32_t, bool, string, DataType
    bool isRange = false;                         // range [min, max] (numbers) or a list of choices
    double min = 0.0, max = 0.0;
    std::vector<std::string> choices;
};

class ValueRangeDictionary {
public:
    void setRange(const std::string& name, const std::string& type, double min, double max, const std::string& def,
                  const std::string& label);
    void setChoices(const std::string& name, const std::string& type, const std::vector<std::string>& choices,
                    const std::string& def, const std::string& label);
    const ParamSpec* find(const std::string& name) const;
    const std::vector<ParamSpec>& all() const { return m_specs; }

private:
    std::vector<ParamSpec> m_specs;
};

class ConfigurationDictionary {
public:
    // Validates `value` against the spec; an invalid value stores the default and returns false.
    bool set(const ParamSpec& spec, const std::string& value, std::string* why);
    const std::string& get(const std::string& name) const;
    double getDouble(const std::string& name) const;
    int64_t getInt(const std::string& name) const;
    bool getBool(const std::string& name) const;
    DataType getDataType(const std::string& name) const;

private:
    std::map<std::string, std::string> m_values;
};

// Host copy of the receive geometry (RxBeamformerParameters); its identity marks a geometry change.
struct Geometry {
    sb_geometry g{};
    std::vector<float> elementX, elementY, depths;
    std::vector<sb_scanline_rx> scanlines;
    std::vector<int32_t> elementToChannel;
    static std::shared_ptr<const Geometry> copyOf(const sb_geometry& src);
};

struct ImageProperties {
    enum class State { Raw, RawDelayed, RF, EnvDetected, LogCompressed, ScanConverted };
    State state = State::Raw;
    std::shared_ptr<const Geometry> geometry;  // scanline grid and depths (scan conversion)
    uint32_t numScanlines = 0, numSamples = 0;
    uint32_t layoutX = 1, layoutY = 1;
    double depthMM = 0.0;
    double imageResolutionMM = 0.1;
    std::map<std::string, std::string> specific;  // setSpecificParameter
};

enum class RecordType { RawData, Image };

struct RecordObject {
    virtual ~RecordObject() = default;
    virtual RecordType getType() const = 0;
    std::shared_ptr<const ImageProperties> properties;
    sb_stream stream = nullptr;
};

// Channel data [tx][channel][sample] (state Raw) or raw-delayed data [scanline][channel][depth].
struct USRawData : RecordObject {
    RecordType getType() const override { return RecordType::RawData; }
    std::shared_ptr<const Geometry> geometry;
    std::shared_ptr<void> data;  // device memory (owned, or a non-owning alias)
    DataType dtype = DataType::Int16;
    uint32_t numTx = 0, numChannels = 0, numSamples = 0;
};

// Image [size[1] samples][size[0] scanlines] (x fastest), or a scan-converted image / volume.
struct USImage : RecordObject {
    RecordType getType() const override { return RecordType::Image; }
    uint32_t size[3] = {0, 0, 1};
    std::shared_ptr<void> data;
    DataType dtype = DataType::Float;
};

// Device buffer allocated and freed in stream order.
std::shared_ptr<void> deviceBuffer(size_t bytes, sb_stream stream);

class AbstractNode {
public:
    explicit AbstractNode(std::string nodeID) : m_nodeID(std::move(nodeID)) {}
    virtual ~AbstractNode() = default;
    AbstractNode(const AbstractNode&) = delete;
    AbstractNode& operator=(const AbstractNode&) = delete;

    const std::string& getNodeID() const { return m_nodeID; }
    virtual const char* getType() const = 0;
    size_t getNumInputs() const { return 1; }
    size_t getNumOutputs() const { return 1; }
    const ValueRangeDictionary& getValueRangeDictionary() const { return m_valueRangeDictionary; }

    // Configuration entry change (validated; returns false and keeps the default if invalid).
    bool setParameter(const std::string& name, const std::string& value);
    std::string getParameter(const std::string& name) const;
    // Processes one record; nullptr on a type / state mismatch or a failed call (see lastError()).
    std::shared_ptr<RecordObject> process(const std::shared_ptr<RecordObject>& in);
    std::string lastError() const;

protected:
    // Call at the end of a derived constructor: fills the defaults, then configurationChanged().
    void finishConstruction();
    virtual void configurationChanged() = 0;
    virtual void configurationEntryChanged(const std::string& /*key*/) { configurationChanged(); }
    virtual std::shared_ptr<RecordObject> processLocked(const std::shared_ptr<RecordObject>& in) = 0;
    std::shared_ptr<RecordObject> fail(const std::string& why);

    ValueRangeDictionary m_valueRangeDictionary;
    ConfigurationDictionary m_configurationDictionary;
    mutable std::mutex m_mutex;

private:
    std::string m_nodeID;
    std::string m_lastError;
};

// InterfaceFactory::createNode analogue (SupraLib/InterfaceFactory.cpp:212-251) for the receive-path
// types: BeamformingNode, RawDelayNode, BeamformingMVNode, HilbertFirEnvelopeNode,
// IQDemodulatorNode, LogCompressorNode, ScanConverterNode, TemporalFilterNode, BeamformingMVpcgNode,
// HilbertEnvelopeNode. nullptr for other types.
std::unique_ptr<AbstractNode> createNode(const std::string& type, const std::string& nodeID);
std::vector<std::string> nodeTypes();

class Graph {
public:
    // Parses the XML text; nodes of unknown types are an error unless listed as inputs or as types
    // outside the receive path (returned by skippedNodes(), bypassed in the chain).
    static std::unique_ptr<Graph> fromXml(const std::string& xml, std::string* error);
    AbstractNode* node(const std::string& id) const;
    const std::vector<std::string>& chain() const { return m_chain; }    // node IDs in processing order
    const std::vector<std::string>& skippedNodes() const { return m_skipped; }
    // Pushes `in` from the first node after the input through the chain; returns the last output.
    std::shared_ptr<RecordObject> process(const std::shared_ptr<RecordObject>& in, std::string* error);
    const std::string& inputType() const { return m_inputType; }
    // a parameter of the first input ("" if absent)
    std::string inputParam(const std::string& name) const {
        auto it = m_inputParams.find(name);
        return it == m_inputParams.end() ? std::string() : it->second;
    }

private:
    std::map<std::string, std::unique_ptr<AbstractNode>> m_nodes;
    std::vector<std::string> m_chain, m_skipped;
    std::string m_inputType;                            // type of the first <input>
    std::map<std::string, std::string> m_inputParams;  // its <param> values
};

}  // namespace supra_b200
