// RVS configuration front end.  The JSON grammar and the validation rules
// follow rvs/src/JsonParser.cpp, rvs/src/Parameters.cpp, rvs/src/Config.cpp
// and rvs/src/PoseTraces.cpp; the code is an independent implementation.
#include "frontend.hpp"

#include <cctype>
#include <cmath>
#include <fstream>
#include <regex>
#include <sstream>

namespace rvsb {
namespace json {
namespace {

struct Reader {
    const std::string& s;
    size_t i = 0;

    int peek() const { return i < s.size() ? (unsigned char)s[i] : -1; }
    int get() { return i < s.size() ? (unsigned char)s[i++] : -1; }
    void ws() {
        while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    }
    void expect(int c) {
        int a = get();
        if (a != c) {
            std::ostringstream what;
            what << "Expected '" << (char)c << "' but found '" << (char)a << "'";
            throw ConfigError(what.str());
        }
    }

    ValuePtr value() {
        ws();
        int c = peek();
        auto v = std::make_shared<Value>();
        if (c == '{') {
            v->type = Value::Type::object;
            get();
            ws();
            bool first = true;
            while (peek() != '}') {
                if (!first) {
                    expect(',');
                    ws();
                }
                first = false;
                std::string key = string_lit();
                ws();
                expect(':');
                ws();
                v->object[key] = value();
                ws();
                if (peek() == -1) throw ConfigError("Unexpected end of JSON object");
            }
            get();
        } else if (c == '[') {
            v->type = Value::Type::array;
            get();
            ws();
            if (peek() != ']') {
                v->array.push_back(value());
                ws();
                while (peek() == ',') {
                    get();
                    v->array.push_back(value());
                    ws();
                }
            }
            expect(']');
        } else if (c == '"') {
            v->type = Value::Type::string;
            v->string = string_lit();
        } else if (c == 't' || c == 'f') {
            v->type = Value::Type::boolean;
            v->boolean = c == 't';
            for (char ch : std::string(v->boolean ? "true" : "false")) expect(ch);
        } else if (c == 'n') {
            for (char ch : std::string("null")) expect(ch);
        } else if (c == '-' || (c >= 0 && std::isdigit(c))) {
            v->type = Value::Type::number;
            size_t used = 0;
            try {
                v->number = std::stod(s.substr(i, 64), &used);
            } catch (const std::exception&) {
                throw ConfigError("Invalid JSON number");
            }
            i += used;
        } else {
            std::ostringstream what;
            what << "Invalid character " << (char)c;
            throw ConfigError(what.str());
        }
        return v;
    }

    std::string string_lit() {
        expect('"');
        std::string out;
        for (;;) {
            int c = get();
            if (c == -1) throw ConfigError("Unterminated JSON string");
            if (c == '"') break;
            if (c == '\\') throw ConfigError("JSON parser: string escaping not implemented");
            out.push_back((char)c);
        }
        return out;
    }
};

}  // namespace

Node Node::parse(const std::string& text) {
    Reader r{text};
    try {
        auto v = r.value();
        r.ws();
        if (r.peek() != -1) throw ConfigError(std::string("Stray character ") + (char)r.peek());
        return Node(v);
    } catch (const ConfigError& e) {
        throw ConfigError(std::string("JSON parser: ") + e.what());
    }
}

Node Node::optional(const std::string& key) const {
    if (overrides_) {
        auto it = overrides_->object.find(key);
        if (it != overrides_->object.end()) return Node(it->second);
    }
    if (v_->type != Value::Type::object)
        throw ConfigError("JSON parser: Querying optional key '" + key + "', but node is not an object");
    auto it = v_->object.find(key);
    if (it == v_->object.end()) return Node();
    return Node(it->second);
}

Node Node::require(const std::string& key) const {
    Node n = optional(key);
    if (!n) throw ConfigError("JSON parser: Parameter " + key + " is required but missing");
    return n;
}

Node Node::at(size_t i) const {
    if (v_->type != Value::Type::array) throw ConfigError("JSON parser: Expected an array");
    if (i >= v_->array.size()) throw ConfigError("JSON parser: array index out of range");
    return Node(v_->array[i]);
}

size_t Node::size() const {
    if (v_->type == Value::Type::array) return v_->array.size();
    if (v_->type == Value::Type::object) return v_->object.size();
    throw ConfigError("JSON parser: Expected an array or object");
}

double Node::asDouble() const {
    if (v_->type != Value::Type::number) throw ConfigError("JSON parser: Expected a number");
    return v_->number;
}

// JsonParser.cpp:303-314: rounds to nearest and rejects only a positive
// rounding error above 1e-6.
int Node::asInt() const {
    double value = asDouble();
    int rounded = static_cast<int>(std::lround(value));
    double error = value - rounded;
    if (error > 1e-6) throw ConfigError("JSON parser: Expected an integer value");
    return rounded;
}

const std::string& Node::asString() const {
    if (v_->type != Value::Type::string) throw ConfigError("JSON parser: Expected a string");
    return v_->string;
}

bool Node::asBool() const {
    if (v_->type != Value::Type::boolean) throw ConfigError("JSON parser: Expected a boolean");
    return v_->boolean;
}

Node::operator bool() const {
    if (v_->type == Value::Type::null) return false;
    if (v_->type == Value::Type::boolean) return v_->boolean;
    return true;
}

}  // namespace json

namespace {

template <int N>
void float_vec(const json::Node& n, float* out) {
    if (n.size() != (size_t)N) throw ConfigError("JSON parser: Expected a vector of floats");
    for (int k = 0; k < N; ++k) out[k] = n.at(k).asFloat();
}

template <int N>
void int_vec(const json::Node& n, int* out) {
    if (n.size() != (size_t)N) throw ConfigError("JSON parser: Expected a vector of floats");
    for (int k = 0; k < N; ++k) out[k] = n.at(k).asInt();
}

}  // namespace

rvsb_camera parse_camera(const json::Node& root, CropRegion* crop) {
    rvsb_camera c{};
    const std::string& proj = root.require("Projection").asString();
    if (proj == "Perspective")
        c.projection = RVSB_PROJ_PERSPECTIVE;
    else if (proj == "Equirectangular")
        c.projection = RVSB_PROJ_EQUIRECTANGULAR;
    else
        throw ConfigError("Unknown projection type \"" + proj + "\"");
    float_vec<3>(root.require("Position"), c.position);
    float_vec<3>(root.require("Rotation"), c.rotation);
    float_vec<2>(root.require("Depth_range"), c.depth_range);
    if (!(c.depth_range[0] < c.depth_range[1]))
        throw ConfigError("Inverted depth range: [near, far] with near > far is not allowed");
    if (c.depth_range[1] > 1000.f)
        throw ConfigError(
            "Invalid depth range: [near, far] with far > 1000 is not allowed because 1000 stands for infinity.");
    c.has_invalid_depth = 1;
    if (auto n = root.optional("HasInvalidDepth")) c.has_invalid_depth = n.asBool() ? 1 : 0;
    int res[2];
    int_vec<2>(root.require("Resolution"), res);
    c.width = res[0];
    c.height = res[1];
    c.bit_depth_color = root.require("BitDepthColor").asInt();
    c.bit_depth_depth = root.require("BitDepthDepth").asInt();
    if (root.require("ColorSpace").asString() != "YUV420")
        throw ConfigError("This version of RVS only supports YUV420 color space for texture");
    const std::string& dcs = root.require("DepthColorSpace").asString();
    if (dcs == "YUV420")
        c.depth_color_format = RVSB_FMT_YUV420;
    else if (dcs == "YUV400")
        c.depth_color_format = RVSB_FMT_YUV400;
    else
        throw ConfigError("This version of RVS only supports YUV420 and YUV400 color space for depth");
    if (c.projection == RVSB_PROJ_EQUIRECTANGULAR) {
        float_vec<2>(root.require("Hor_range"), c.hor_range);
        c.full_hor_range = 0;
        try {
            int hr[2];
            int_vec<2>(root.require("Hor_range"), hr);
            c.full_hor_range = (hr[0] == -180 && hr[1] == 180) ? 1 : 0;
        } catch (const ConfigError&) {
        }
        float_vec<2>(root.require("Ver_range"), c.ver_range);
    }
    CropRegion cr;
    cr.w = cr.padded_w = c.width;
    cr.h = cr.padded_h = c.height;
    if (auto n = root.optional("Crop_region")) {
        int v[4];
        int_vec<4>(n, v);
        if (v[0] != 0 || v[1] != 0 || v[2] != c.width || v[3] != c.height) {
            if (!crop) throw Unsupported("Crop_region needs the camera's padded resolution reported beside it");
            if (v[0] < 0 || v[1] < 0 || v[2] <= 0 || v[3] <= 0 || v[0] > c.width - v[2] || v[1] > c.height - v[3])
                throw ConfigError("Crop_region must lie inside the resolution");
            cr.x = v[0];
            cr.y = v[1];
            cr.w = v[2];
            cr.h = v[3];
        }
    }
    c.width = cr.w;
    c.height = cr.h;
    if (c.projection == RVSB_PROJ_PERSPECTIVE) {
        float_vec<2>(root.require("Focal"), c.focal);
        float_vec<2>(root.require("Principle_point"), c.principle_point);
        c.principle_point[0] -= (float)cr.x;
        c.principle_point[1] -= (float)cr.y;
    }
    if (crop) *crop = cr;
    if (auto n = root.optional("DisplacementMethod")) {
        if (n.asString() == "Polynomial") throw Unsupported("Polynomial displacement is not supported");
    }
    if (auto n = root.optional("Multi_depth_range")) {
        float md[2];
        float_vec<2>(n, md);
        if (!(md[0] < md[1]))
            throw ConfigError("Inverted depth range: [near, far] with near > far is not allowed");
    }
    if (root.require("Depthmap").asInt() != 1)
        throw ConfigError("This version of RVS only supports Depthmap 1");
    root.require("Background").asInt();
    if (c.width <= 0 || c.height <= 0) throw ConfigError("Resolution must be positive");
    if (c.bit_depth_color < 1 || c.bit_depth_color > 16 || c.bit_depth_depth < 1 || c.bit_depth_depth > 16)
        throw ConfigError("invalid raw image bit depth");
    return c;
}

std::vector<Pose> parse_pose_trace(const std::string& text) {
    std::istringstream stream(text);
    std::string line;
    std::getline(stream, line);
    static const std::regex re_header("\\s*X\\s*,\\s*Y\\s*,\\s*Z\\s*,\\s*Yaw\\s*,\\s*Pitch\\s*,\\s*Roll\\s*");
    if (!std::regex_match(line, re_header)) throw ConfigError("Format error in the pose trace header");
    static const std::regex re_row("([^,]+),([^,]+),([^,]+),([^,]+),([^,]+),([^,]+)");
    static const std::regex re_empty("\\s*");
    std::vector<Pose> trace;
    bool trailing_empty = false;
    while (std::getline(stream, line)) {
        std::smatch m;
        if (!trailing_empty && std::regex_match(line, m, re_row)) {
            Pose p;
            try {
                for (int k = 0; k < 3; ++k) p.position[k] = std::stof(m[1 + k].str());
                for (int k = 0; k < 3; ++k) p.rotation[k] = std::stof(m[4 + k].str());
            } catch (const std::exception&) {
                throw ConfigError("Format error in a pose trace row");
            }
            trace.push_back(p);
        } else if (std::regex_match(line, re_empty)) {
            trailing_empty = true;
        } else {
            throw ConfigError("Format error in a pose trace row");
        }
    }
    return trace;
}

std::string read_text_file(const std::string& path, const char* what) {
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) throw IoError(std::string("Failed to open ") + what + " \"" + path + "\" for reading");
    std::ostringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

namespace {

// Config::loadCamerasParametersFromFile (Config.cpp:122-175).
std::vector<rvsb_camera> load_cameras(const std::string& path, const std::vector<std::string>& names,
                                      const json::Node& overrides, std::vector<CropRegion>& crops) {
    json::Node root = json::Node::parse(read_text_file(path, "camera parameters file"));
    std::string version = root.require("Version").asString();
    std::string v2 = version.substr(0, 2);
    if (v2 != "2." && v2 != "3." && v2 != "4.")
        throw ConfigError("Version of the camera parameters file is not compatible with this version of RVS");
    std::map<std::string, std::pair<rvsb_camera, CropRegion>> index;
    json::Node cams = root.require("cameras");
    for (size_t i = 0; i < cams.size(); ++i) {
        json::Node node = cams.at(i);
        std::string name = node.require("Name").asString();
        if (index.count(name)) throw ConfigError("Camera parameters file has duplicate camera '" + name + "'");
        if (overrides) node.setOverrides(overrides);
        CropRegion cr;
        const rvsb_camera c = parse_camera(node, &cr);
        index.emplace(name, std::make_pair(c, cr));
    }
    std::vector<rvsb_camera> out;
    for (const auto& n : names) {
        auto it = index.find(n);
        if (it == index.end()) throw ConfigError("Camera parameters file does not have camera '" + n + "'");
        out.push_back(it->second.first);
        crops.push_back(it->second.second);
    }
    return out;
}

std::vector<std::string> string_list(const json::Node& n) {
    std::vector<std::string> v;
    for (size_t i = 0; i < n.size(); ++i) v.push_back(n.at(i).asString());
    return v;
}

}  // namespace

Config load_config(const std::string& path) {
    json::Node root = json::Node::parse(read_text_file(path, "configuration file"));
    Config c;
    c.version = root.require("Version").asString();
    if (c.version.substr(0, 2) != "2." && c.version.substr(0, 2) != "3.")
        throw ConfigError("Configuration file does not match the RVS version");
    c.input_names = string_list(root.require("InputCameraNames"));
    c.virtual_names = string_list(root.require("VirtualCameraNames"));
    c.params_real = load_cameras(root.require("InputCameraParameterFile").asString(), c.input_names,
                                 root.optional("InputOverrides"), c.crop_real);
    c.params_virtual = load_cameras(root.require("VirtualCameraParameterFile").asString(), c.virtual_names,
                                    root.optional("VirtualOverrides"), c.crop_virtual);
    auto inputs = [&](const char* key, std::vector<std::string>& dst) {
        json::Node n = root.require(key);
        if (n.size() != c.input_names.size())
            throw ConfigError(std::string("Length of ") + key + " should match with InputCameraNames");
        dst = string_list(n);
    };
    inputs("ViewImageNames", c.texture_names);
    inputs("DepthMapNames", c.depth_names);
    auto outputs = [&](const char* key, std::vector<std::string>& dst) {
        if (json::Node n = root.optional(key)) {
            if (n.size() != c.virtual_names.size())
                throw ConfigError(std::string("Length of ") + key + " should match with VirtualCameraNames");
            dst = string_list(n);
        }
    };
    outputs("OutputFiles", c.outfilenames);
    outputs("MaskedOutputFiles", c.outmaskedfilenames);
    outputs("OutputMasks", c.outmaskfilenames);
    outputs("DepthOutputFiles", c.outdepthfilenames);
    outputs("MaskedDepthOutputFiles", c.outmaskdepthfilenames);
    if (auto n = root.optional("ValidityThreshold")) c.validity_threshold = (float)n.asDouble();
    if (auto n = root.optional("ViewSynthesisMethod")) c.vs_method = n.asString();
    if (c.vs_method != "Triangles") throw ConfigError("Unknown view synthesis method \"" + c.vs_method + "\"");
    if (auto n = root.optional("BlendingMethod")) c.blending_method = n.asString();
    if (auto n = root.optional("BlendingFactor")) c.blending_factor = (float)n.asDouble();
    if (c.blending_method == "Multispectral") {
        c.blending_low_freq_factor = (float)root.require("BlendingLowFreqFactor").asDouble();
        c.blending_high_freq_factor = (float)root.require("BlendingHighFreqFactor").asDouble();
    }
    if (c.blending_method != "Simple")
        throw ConfigError("Unknown view blending method \"" + c.blending_method + "\"");
    if (auto n = root.optional("StartFrame")) c.start_frame = n.asInt();
    if (auto n = root.optional("NumberOfFrames")) c.number_of_frames = n.asInt();
    if (auto n = root.optional("NumberOfOutputFrames"))
        c.number_of_output_frames = n.asInt();
    else
        c.number_of_output_frames = c.number_of_frames;
    if (auto n = root.optional("Precision")) c.precision = (float)n.asDouble();
    if (!std::isfinite(c.precision) || !(c.precision > 0.f)) throw ConfigError("Precision must be positive");
    if (auto n = root.optional("ColorSpace")) {
        const std::string& cs = n.asString();
        if (cs != "YUV" && cs != "RGB") throw ConfigError("Unknown color space");
    }
    if (auto n = root.optional("VirtualPoseTraceName")) {
        std::string fp = n.asString();
        if (!fp.empty()) {
            c.pose_trace = parse_pose_trace(read_text_file(fp, "pose trace"));
            if ((size_t)(c.start_frame + c.number_of_frames) > c.pose_trace.size())
                throw ConfigError(
                    "Error: Number of frames to process is larger then number of entries in pose trace file");
        }
    }
    return c;
}

}  // namespace rvsb
