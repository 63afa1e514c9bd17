// RVS configuration front end: JSON values, camera parameters, RVS config,
// pose trace.  Semantics follow the reference's parser and validation.
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "rvsb.h"

namespace rvsb {

// Error raised for a rejected configuration (maps to RVSB_E_CONFIG).
struct ConfigError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// Valid reference option this build does not implement (RVSB_E_UNSUPPORTED).
struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// File missing or unreadable (RVSB_E_IO).
struct IoError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

namespace json {

struct Value;
using ValuePtr = std::shared_ptr<Value>;

struct Value {
    enum class Type { number, string, array, object, boolean, null };
    Type type = Type::null;
    double number = 0;
    std::string string;
    bool boolean = false;
    std::vector<ValuePtr> array;
    std::map<std::string, ValuePtr> object;
};

// A view on a value with optional overrides (JsonParser.hpp:46-118).
class Node {
public:
    Node() : v_(std::make_shared<Value>()) {}
    explicit Node(ValuePtr v) : v_(std::move(v)) {}
    static Node parse(const std::string& text);

    void setOverrides(const Node& o) { overrides_ = o.v_; }
    Value::Type type() const { return v_->type; }
    Node optional(const std::string& key) const;
    Node require(const std::string& key) const;
    Node at(size_t i) const;
    size_t size() const;
    double asDouble() const;
    float asFloat() const { return static_cast<float>(asDouble()); }
    int asInt() const;
    const std::string& asString() const;
    bool asBool() const;
    explicit operator bool() const;

private:
    ValuePtr v_;
    ValuePtr overrides_;
};

}  // namespace json

// "Crop_region" of a camera (Parameters::setCropRegionFrom,
// Parameters.cpp:424-434): the region x, y, w, h of the padded resolution
// the camera's image covers.  Without the key it is the whole resolution.
struct CropRegion {
    int x = 0, y = 0, w = 0, h = 0;
    int padded_w = 0, padded_h = 0;
};

// Parameters::readFrom (Parameters.cpp:104-129).  With `crop`, a
// Crop_region is applied as the reference's getters do: the camera's size
// is the region's (getSize, Parameters.cpp:187-190) and a perspective
// principal point is moved by the region's top-left corner
// (getPrinciplePoint, Parameters.cpp:245-249); ERP ranges already refer to
// the region.  Without `crop` (a camera parsed alone, with nowhere to
// report its padded resolution), a region other than the whole resolution
// is rejected.
rvsb_camera parse_camera(const json::Node& node, CropRegion* crop = nullptr);

struct Pose {
    float position[3];
    float rotation[3];
};

// PoseTrace::loadFrom (PoseTraces.cpp:54-92).
std::vector<Pose> parse_pose_trace(const std::string& text);

struct Config {
    std::string version;
    std::vector<std::string> input_names, virtual_names;
    std::vector<rvsb_camera> params_real, params_virtual;
    std::vector<CropRegion> crop_real, crop_virtual;
    std::vector<std::string> texture_names, depth_names;
    std::vector<std::string> outfilenames, outmaskedfilenames, outmaskfilenames, outdepthfilenames,
        outmaskdepthfilenames;
    float validity_threshold = 5000.f;
    std::string vs_method = "Triangles";
    std::string blending_method = "Simple";
    float blending_low_freq_factor = 0.f;
    float blending_high_freq_factor = 0.f;
    float blending_factor = 5.f;
    int start_frame = 0;
    int number_of_frames = 1;
    int number_of_output_frames = 1;
    float precision = 1.f;
    std::vector<Pose> pose_trace;
};

// Config::loadFromFile (Config.cpp:72-120).
Config load_config(const std::string& path);

std::string read_text_file(const std::string& path, const char* what);

}  // namespace rvsb
