// Tree files in the reference's gzip-compressed JSON format (RandomTreeExport::writeTree/writeJSON,
// export.cpp:180-313; RandomTreeImport::readTree/readJSON, import.cpp:42-266).
//
// The format is boost::property_tree's JSON: every value is a string, keys containing dots become
// nested objects, XY pairs are two-element arrays. A node holds id, level, samples, leaf, a
// histogram keyed "R,G,B (label)", and for split nodes split.{threshold, score, featureId, feature}
// plus left/right children. The header carries the training configuration and
// classLabelPriorDistribution.{label}. As in the reference, the device list is written as
// "deviceId" but read as "deviceIds" (export.cpp:202 vs import.cpp:244). Floats are written with
// enough digits to round-trip exactly.
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "tree.h"

namespace cf {
namespace {

// ---- minimal JSON value --------------------------------------------------------------------------
struct Json {
    enum Kind { Null, Str, Obj, Arr } kind = Null;
    std::string str;
    std::vector<std::pair<std::string, Json>> items;  // object members or array elements (key "")
    const Json* get(const std::string& k) const {
        for (const auto& kv : items)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
    const Json& at(const std::string& k) const {
        const Json* j = get(k);
        if (!j) fail(CF_ERR_IO, "tree file: missing key '" + k + "'");
        return *j;
    }
};

class Parser {
public:
    explicit Parser(const std::string& s) : s_(s) {}
    Json parse() {
        Json v = value();
        ws();
        if (i_ != s_.size()) fail(CF_ERR_IO, "tree file: trailing characters");
        return v;
    }

private:
    const std::string& s_;
    size_t i_ = 0;
    void ws() {
        while (i_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[i_]))) i_++;
    }
    char peek() {
        ws();
        if (i_ >= s_.size()) fail(CF_ERR_IO, "tree file: unexpected end");
        return s_[i_];
    }
    void expect(char c) {
        if (peek() != c) fail(CF_ERR_IO, std::string("tree file: expected '") + c + "'");
        i_++;
    }
    std::string string() {
        expect('"');
        std::string out;
        while (i_ < s_.size() && s_[i_] != '"') {
            char c = s_[i_++];
            if (c == '\\') {
                if (i_ >= s_.size()) break;
                const char e = s_[i_++];
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (i_ + 4 > s_.size()) fail(CF_ERR_IO, "tree file: bad escape");
                        const unsigned code = static_cast<unsigned>(std::stoul(s_.substr(i_, 4), nullptr, 16));
                        i_ += 4;
                        out += static_cast<char>(code < 128 ? code : '?');
                        break;
                    }
                    default: out += e;
                }
            } else {
                out += c;
            }
        }
        expect('"');
        return out;
    }
    Json value() {
        const char c = peek();
        Json v;
        if (c == '{') {
            i_++;
            v.kind = Json::Obj;
            if (peek() == '}') {
                i_++;
                return v;
            }
            for (;;) {
                std::string k = string();
                expect(':');
                v.items.emplace_back(std::move(k), value());
                if (peek() == ',') {
                    i_++;
                    continue;
                }
                expect('}');
                return v;
            }
        }
        if (c == '[') {
            i_++;
            v.kind = Json::Arr;
            if (peek() == ']') {
                i_++;
                return v;
            }
            for (;;) {
                v.items.emplace_back(std::string(), value());
                if (peek() == ',') {
                    i_++;
                    continue;
                }
                expect(']');
                return v;
            }
        }
        if (c == '"') {
            v.kind = Json::Str;
            v.str = string();
            return v;
        }
        // bare literal (numbers, true/false/null written by other JSON writers)
        const size_t b = i_;
        while (i_ < s_.size() && s_[i_] != ',' && s_[i_] != '}' && s_[i_] != ']' &&
               !std::isspace(static_cast<unsigned char>(s_[i_])))
            i_++;
        v.kind = Json::Str;
        v.str = s_.substr(b, i_ - b);
        return v;
    }
};

long long as_int(const Json& j) {
    try {
        return std::stoll(j.str);
    } catch (...) {
        fail(CF_ERR_IO, "tree file: not an integer: '" + j.str + "'");
    }
}
double as_double(const Json& j) {
    try {
        return std::stod(j.str);
    } catch (...) {
        fail(CF_ERR_IO, "tree file: not a number: '" + j.str + "'");
    }
}
bool as_bool(const Json& j) { return j.str == "true" || j.str == "1"; }

// ---- writer ---------------------------------------------------------------------------------------
std::string quote(const std::string& s) {
    std::string o = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        if (c == '/') {
            o += "\\/";
            continue;
        }
        o += c;
    }
    return o + "\"";
}

std::string fmt_float(float v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.9g", static_cast<double>(v));
    return b;
}
std::string fmt_double(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

// Colour of a label for histogram keys. Labels are dense indices of a colour registry in the
// reference (LabelImage::encodeColor, image.cpp:664-673); without a registry a fixed palette is used.
std::string label_color(int label) {
    const int r = (label * 67 + 13) % 256, g = (label * 131 + 71) % 256, b = (label * 29 + 199) % 256;
    return std::to_string(r) + "," + std::to_string(g) + "," + std::to_string(b);
}

class Writer {
public:
    explicit Writer(bool verbose) : verbose_(verbose) {}
    std::string out;
    void open() { out += "{\n"; depth_++; first_ = true; }
    void close() { depth_--; out += "\n" + indent() + "}"; first_ = false; }
    void key(const std::string& k) {
        if (!first_) out += ",\n";
        out += indent() + quote(k) + ": ";
        first_ = true;
    }
    void kv(const std::string& k, const std::string& v) {
        key(k);
        out += quote(v);
        first_ = false;
    }
    void array(const std::string& k, const std::vector<std::string>& vals) {
        key(k);
        out += "[";
        for (size_t i = 0; i < vals.size(); i++) out += (i ? "," : "") + quote(vals[i]);
        out += "]";
        first_ = false;
    }
    void node(const cf_tree& t, int i) {
        const int C = t.C;
        open();
        kv("id", std::to_string(t.tree_id + i));
        kv("level", std::to_string(t.level[i]));
        kv("samples", std::to_string(t.nsamp[i]));
        kv("leaf", t.left[i] < 0 ? "true" : "false");
        key("histogram");
        open();
        for (int c = 0; c < C; c++)
            kv(label_color(c) + " (" + std::to_string(c) + ")", std::to_string(t.hist[static_cast<size_t>(i) * C + c]));
        close();
        if (t.left[i] >= 0) {
            const int8_t* f = &t.feature[static_cast<size_t>(i) * 11];
            key("split");
            open();
            kv("threshold", fmt_float(t.threshold[i]));
            kv("score", fmt_double(t.score[i]));
            kv("featureId", std::to_string(t.feature_id[i]));
            key("feature");
            open();
            kv("type", f[0] == 0 ? "depth" : "color");
            if (f[0] != 0) {
                kv("channel1", std::to_string(static_cast<uint8_t>(f[9])));
                kv("channel2", std::to_string(static_cast<uint8_t>(f[10])));
            }
            array("offset1", {std::to_string(f[1]), std::to_string(f[2])});
            array("region1", {std::to_string(f[5]), std::to_string(f[6])});
            array("offset2", {std::to_string(f[3]), std::to_string(f[4])});
            array("region2", {std::to_string(f[7]), std::to_string(f[8])});
            close();
            close();
            key("left");
            node(t, t.left[i]);
            first_ = false;
            key("right");
            node(t, t.left[i] + 1);
            first_ = false;
        }
        close();
    }

private:
    bool verbose_;
    int depth_ = 0;
    bool first_ = true;
    std::string indent() const { return std::string(4 * depth_, ' '); }
};

// /proc/cpuinfo as "key: value" records, one per logical processor (the fields the reference's
// header keys numPhysicalCPUs and processorModels are taken from, export.cpp:91-177).
std::vector<std::map<std::string, std::string>> cpu_records() {
    std::vector<std::map<std::string, std::string>> recs;
    FILE* f = std::fopen("/proc/cpuinfo", "r");
    if (!f) return recs;
    auto trim = [](const std::string& v) {
        const size_t a = v.find_first_not_of(" \t\r\n"), b = v.find_last_not_of(" \t\r\n");
        return a == std::string::npos ? std::string() : v.substr(a, b - a + 1);
    };
    char line[4096];
    while (std::fgets(line, sizeof line, f)) {
        const std::string l(line);
        const size_t colon = l.find(':');
        if (colon == std::string::npos) continue;
        const std::string k = trim(l.substr(0, colon)), v = trim(l.substr(colon + 1));
        if (k == "processor" || recs.empty()) recs.emplace_back();   // "processor" opens a record
        if (!v.empty()) recs.back()[k] = v;
    }
    std::fclose(f);
    return recs;
}

const char* mode_string(int m) { return m == 0 ? "cpu" : (m == 2 ? "compare" : "gpu"); }
int parse_mode(const std::string& s) {
    if (s == "cpu") return 0;
    if (s == "gpu") return 1;
    if (s == "compare") return 2;
    fail(CF_ERR_IO, "illegal acceleration mode: " + s);
}

std::string read_file(const char* path) {
    gzFile f = gzopen(path, "rb");
    if (!f) fail(CF_ERR_IO, std::string("failed to read tree file: '") + path + "'");
    std::string data;
    char buf[1 << 16];
    int n;
    while ((n = gzread(f, buf, sizeof buf)) > 0) data.append(buf, n);
    int err = 0;
    const char* msg = gzerror(f, &err);
    gzclose(f);
    if (n < 0 || (err != Z_OK && err != Z_STREAM_END)) fail(CF_ERR_IO, std::string("gzip read error: ") + msg);
    return data;
}

// readTree (import.cpp:96-160): node ids must form the breadth-first numbering the packer expects.
void read_node(const Json& j, int tree_id, cf_tree& t, int parent_level, int index) {
    const long long id = as_int(j.at("id"));
    if (id - tree_id != index) fail(CF_ERR_IO, "tree file: node ids are not in breadth-first order");
    t.level[index] = static_cast<int32_t>(as_int(j.at("level")));
    (void)parent_level;
    t.nsamp[index] = static_cast<uint32_t>(as_int(j.at("samples")));
    const Json& h = j.at("histogram");
    std::vector<uint32_t> hist(t.C, 0);
    uint64_t sum = 0;
    for (const auto& kv : h.items) {
        const std::string& k = kv.first;
        const size_t start = k.find(" (");
        const size_t stop = k.find(')', start);
        if (start == std::string::npos || stop == std::string::npos)
            fail(CF_ERR_IO, "failed to parse histogram key: '" + k + "'");
        const int label = std::stoi(k.substr(start + 2, stop - start - 2));
        if (label < 0 || label >= t.C) fail(CF_ERR_IO, "histogram label out of range in key '" + k + "'");
        hist[label] = static_cast<uint32_t>(as_int(kv.second));
        sum += hist[label];
    }
    if (sum < t.nsamp[index]) fail(CF_ERR_IO, "incorrect histogram sum");
    std::memcpy(&t.hist[static_cast<size_t>(index) * t.C], hist.data(), 4 * t.C);
    std::memset(&t.feature[static_cast<size_t>(index) * 11], 0, 11);
    t.left[index] = -1;
    t.threshold[index] = std::nanf("");
    t.score[index] = std::nan("");
    t.feature_id[index] = -1;
}

}  // namespace
}  // namespace cf

using namespace cf;

extern "C" {

cf_status cf_tree_write_json(cf_tree* tree, const cf_train_config* config, const uint32_t* prior, const char* path,
                             int verbose) {
    return guard([&] {
        CF_REQUIRE(tree && config && path, "cf_tree_write_json: NULL argument");
        Writer w(verbose != 0);
        w.open();
        char host[256] = {0};
        gethostname(host, sizeof host - 1);
        w.kv("hostname", host);
        w.kv("buildType", "RELEASE");
        w.kv("version", cf_version());
        std::time_t now = std::time(nullptr);
        char date[64];
        std::strftime(date, sizeof date, "%Y-%b-%d %H:%M:%S", std::gmtime(&now));
        w.kv("date", date);
        w.kv("randomSeed", std::to_string(config->random_seed));
        w.kv("folderTraining", "");
        // host description keys of the reference header (export.cpp:198-200)
        const auto cpus = cpu_records();
        int physical = 0;
        std::vector<std::string> models;
        for (const auto& r : cpus) {
            auto it = r.find("physical id");
            if (it != r.end()) physical = std::max(physical, std::atoi(it->second.c_str()) + 1);
            it = r.find("model name");
            if (it != r.end() && std::find(models.begin(), models.end(), it->second) == models.end())
                models.push_back(it->second);
        }
        std::sort(models.begin(), models.end());
        w.kv("numCores", std::to_string(std::max(1L, sysconf(_SC_NPROCESSORS_ONLN))));
        w.kv("numPhysicalCPUs", std::to_string(physical));
        w.array("processorModels", models);
        w.kv("accelerationMode", mode_string(config->acceleration_mode));
        w.array("deviceId", {"0"});
        w.kv("samplesPerImage", std::to_string(config->samples_per_image));
        w.kv("featureCount", std::to_string(config->feature_count));
        w.kv("thresholds", std::to_string(config->thresholds));
        w.kv("boxRadius", std::to_string(config->box_radius));
        w.kv("regionSize", std::to_string(config->region_size));
        w.kv("maxDepth", std::to_string(config->max_depth));
        w.kv("numThreads", std::to_string(config->num_threads));
        w.kv("minSampleCount", std::to_string(config->min_sample_count));
        w.kv("maxSamplesPerBatch", std::to_string(config->max_samples_per_batch));
        w.kv("maxImages", std::to_string(config->max_images));
        w.kv("imageCacheSize", std::to_string(config->image_cache_size));
        w.kv("subsamplingType", config->subsampling_type == 1 ? "pixelUniform" : "classUniform");
        w.kv("useCIELab", config->use_cie_lab ? "true" : "false");
        w.kv("useDepthFilling", config->use_depth_filling ? "true" : "false");
        w.kv("useDepthImages", config->use_depth_images ? "true" : "false");
        w.array("ignoredColors", {});
        const uint32_t* pr = prior ? prior : (tree->prior.empty() ? nullptr : tree->prior.data());
        w.key("classLabelPriorDistribution");
        w.open();
        for (int c = 0; c < tree->C; c++) w.kv(std::to_string(c), std::to_string(pr ? pr[c] : 0));
        w.close();
        w.key("tree");
        w.node(*tree, 0);
        w.close();
        w.out += "\n";
        gzFile f = gzopen(path, "wb");
        if (!f) fail(CF_ERR_IO, std::string("cannot write '") + path + "'");
        const int n = gzwrite(f, w.out.data(), static_cast<unsigned>(w.out.size()));
        const int rc = gzclose(f);
        if (n != static_cast<int>(w.out.size()) || rc != Z_OK) fail(CF_ERR_IO, std::string("gzip write failed: ") + path);
    });
}

cf_status cf_tree_read_json(const char* path, cf_train_config* config, uint32_t* prior, int prior_capacity,
                            cf_tree** out) {
    return guard([&] {
        CF_REQUIRE(path && out, "cf_tree_read_json: NULL argument");
        const std::string data = read_file(path);
        const Json root = Parser(data).parse();
        if (config) {
            std::memset(config, 0, sizeof *config);
            config->random_seed = static_cast<int32_t>(as_int(root.at("randomSeed")));
            config->samples_per_image = static_cast<uint32_t>(as_int(root.at("samplesPerImage")));
            config->feature_count = static_cast<uint32_t>(as_int(root.at("featureCount")));
            config->min_sample_count = static_cast<uint32_t>(as_int(root.at("minSampleCount")));
            config->max_depth = static_cast<int32_t>(as_int(root.at("maxDepth")));
            config->box_radius = static_cast<uint16_t>(as_int(root.at("boxRadius")));
            config->region_size = static_cast<uint16_t>(as_int(root.at("regionSize")));
            config->thresholds = static_cast<uint16_t>(as_int(root.at("thresholds")));
            config->num_threads = static_cast<int32_t>(as_int(root.at("numThreads")));
            config->image_cache_size = static_cast<int32_t>(as_int(root.at("imageCacheSize")));
            config->max_samples_per_batch = static_cast<uint32_t>(as_int(root.at("maxSamplesPerBatch")));
            config->acceleration_mode = parse_mode(root.at("accelerationMode").str);
            const Json* v;
            config->use_cie_lab = (v = root.get("useCIELab")) ? as_bool(*v) : 1;
            config->use_depth_filling = (v = root.get("useDepthFilling")) ? as_bool(*v) : 0;
            config->max_images = (v = root.get("maxImages")) ? static_cast<int32_t>(as_int(*v)) : 0;
            config->subsampling_type = ((v = root.get("subsamplingType")) && v->str == "classUniform") ? 0 : 1;
            config->use_depth_images = (v = root.get("useDepthImages")) ? as_bool(*v) : 1;
            config->horizontal_flipping = 0;
        }
        const Json& pj = root.at("classLabelPriorDistribution");
        const Json& tj = root.at("tree");
        const int C = static_cast<int>(tj.at("histogram").items.size());
        CF_REQUIRE(C >= 1 && C <= 256, "tree file: histogram must hold 1..256 classes");
        std::unique_ptr<cf_tree> t(new cf_tree());
        t->tree_id = static_cast<int>(as_int(tj.at("id")));
        t->C = C;
        t->prior.assign(C, 0);
        for (const auto& kv : pj.items) {
            const int label = std::stoi(kv.first);
            if (label >= 0 && label < C) t->prior[label] = static_cast<uint32_t>(as_int(kv.second));
        }
        if (prior) {
            CF_REQUIRE(prior_capacity >= C, "cf_tree_read_json: prior buffer too small");
            std::memcpy(prior, t->prior.data(), 4 * C);
        }
        // breadth-first walk: node index = id - treeId
        std::vector<const Json*> queue{&tj};
        std::vector<int> index{0};
        std::vector<char> seen;   // node indices read (levels may start at 0 in hand-built files)
        int count = 0;
        t->resize(0);
        for (size_t q = 0; q < queue.size(); q++) {
            const Json& j = *queue[q];
            const int i = index[q];
            if (i + 1 > count) {
                count = i + 1;
                t->resize(count);
                seen.resize(count, 0);
            }
            if (seen[i]) fail(CF_ERR_IO, "tree file: node id " + std::to_string(i + t->tree_id) + " appears twice");
            seen[i] = 1;
            read_node(j, t->tree_id, *t, 0, i);
            const Json* l = j.get("left");
            const Json* r = j.get("right");
            if (l && r) {
                const Json& sp = j.at("split");
                const Json& fj = sp.at("feature");
                int8_t* f = &t->feature[static_cast<size_t>(i) * 11];
                const std::string type = fj.at("type").str;
                if (type != "color" && type != "depth") fail(CF_ERR_IO, "illegal feature type: " + type);
                f[0] = type == "depth" ? 0 : 1;
                auto xy = [&](const char* k, int a, int b) {
                    const Json& arr = fj.at(k);
                    if (arr.items.size() != 2) fail(CF_ERR_IO, std::string("unexpected size of ") + k);
                    f[a] = static_cast<int8_t>(as_int(arr.items[0].second));
                    f[b] = static_cast<int8_t>(as_int(arr.items[1].second));
                };
                xy("offset1", 1, 2);
                xy("offset2", 3, 4);
                xy("region1", 5, 6);
                xy("region2", 7, 8);
                f[9] = f[0] == 1 ? static_cast<int8_t>(as_int(fj.at("channel1"))) : 0;
                f[10] = f[0] == 1 ? static_cast<int8_t>(as_int(fj.at("channel2"))) : 0;
                t->threshold[i] = static_cast<float>(as_double(sp.at("threshold")));
                t->score[i] = as_double(sp.at("score"));
                t->feature_id[i] = static_cast<int32_t>(as_int(sp.at("featureId")));
                const int li = static_cast<int>(as_int(l->at("id"))) - t->tree_id;
                const int ri = static_cast<int>(as_int(r->at("id"))) - t->tree_id;
                if (li <= i || ri != li + 1) fail(CF_ERR_IO, "tree file: children must have consecutive ids");
                t->left[i] = li;
                queue.push_back(l);
                index.push_back(li);
                queue.push_back(r);
                index.push_back(ri);
            }
        }
        // every index must have been filled
        for (int i = 0; i < count; i++)
            if (!seen[i]) fail(CF_ERR_IO, "tree file: missing node " + std::to_string(i));
        // re-apply splits (resize during the walk may have reset nothing; values were written in place)
        *out = t.release();
    });
}

}  // extern "C"
