// gvfile.cpp - .gvx / .gvb / .gvp reader and writer (see gvfile.h).
#include "gvfile.h"

#include "../../include/voxviz_b200.h"

#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <utility>

namespace vv {

namespace {

// ---------------------------------------------------------------------------
// A minimal XML token stream: start and end elements with attributes;
// declarations, comments, CDATA, DOCTYPE and character data are skipped.  A
// self-closing element gives a start and then an end token.  The two
// navigation calls behave as the stream reader the reference parses with:
// next_start_element stops at the first start element (true) or end element
// (false); skip_current_element reads to the end of the element whose start
// was read last.
class XmlStream {
public:
    enum Token { kStart, kEnd, kDone, kError };

    explicit XmlStream(std::string text) : s_(std::move(text)) {}
    size_t size() const { return s_.size(); }

    Token next() {
        if (failed_) return kError;
        if (pending_end_) {
            pending_end_ = false;
            open_.pop_back();
            return kEnd;
        }
        for (;;) {
            const size_t lt = s_.find('<', p_);
            if (lt == std::string::npos) {
                if (!open_.empty()) return fail("unexpected end of document inside <" + open_.back() + ">");
                if (!seen_root_) return fail("no root element");
                p_ = s_.size();
                return kDone;
            }
            p_ = lt;
            if (s_.compare(p_, 4, "<!--") == 0) {
                if (!skip_past("-->")) return fail("unterminated comment");
                continue;
            }
            if (s_.compare(p_, 9, "<![CDATA[") == 0) {
                if (!skip_past("]]>")) return fail("unterminated CDATA section");
                continue;
            }
            if (s_.compare(p_, 2, "<?") == 0) {
                if (!skip_past("?>")) return fail("unterminated processing instruction");
                continue;
            }
            if (s_.compare(p_, 2, "<!") == 0) {  // DOCTYPE, with an optional internal subset
                int depth = 0;
                size_t q = p_ + 2;
                for (; q < s_.size(); ++q) {
                    if (s_[q] == '[') ++depth;
                    else if (s_[q] == ']') --depth;
                    else if (s_[q] == '>' && depth <= 0) break;
                }
                if (q >= s_.size()) return fail("unterminated declaration");
                p_ = q + 1;
                continue;
            }
            if (s_.compare(p_, 2, "</") == 0) {
                p_ += 2;
                std::string n = read_name();
                skip_ws();
                if (n.empty() || p_ >= s_.size() || s_[p_] != '>') return fail("malformed end tag");
                ++p_;
                if (open_.empty() || open_.back() != n) return fail("end tag </" + n + "> does not match");
                open_.pop_back();
                name_ = n;
                return kEnd;
            }
            ++p_;
            if (open_.empty() && seen_root_) return fail("extra content at the end of the document");
            name_ = read_name();
            if (name_.empty()) return fail("malformed start tag");
            attrs_.clear();
            for (;;) {
                const bool ws = skip_ws();
                if (p_ >= s_.size()) return fail("unterminated start tag <" + name_ + ">");
                if (s_[p_] == '>') {
                    ++p_;
                    break;
                }
                if (s_.compare(p_, 2, "/>") == 0) {
                    p_ += 2;
                    pending_end_ = true;
                    break;
                }
                if (!ws) return fail("attributes of <" + name_ + "> must be separated by white space");
                std::string an = read_name();
                if (an.empty()) return fail("malformed attribute in <" + name_ + ">");
                skip_ws();
                if (p_ >= s_.size() || s_[p_] != '=') return fail("attribute " + an + " has no value");
                ++p_;
                skip_ws();
                if (p_ >= s_.size() || (s_[p_] != '"' && s_[p_] != '\'')) return fail("attribute value not quoted");
                const char quote = s_[p_++];
                const size_t end = s_.find(quote, p_);
                if (end == std::string::npos) return fail("unterminated attribute value");
                std::string v;
                if (!decode(s_.substr(p_, end - p_), v)) return fail("bad character reference in " + an);
                p_ = end + 1;
                for (const auto& a : attrs_)
                    if (a.first == an) return fail("attribute " + an + " repeated");
                attrs_.emplace_back(std::move(an), std::move(v));
            }
            open_.push_back(name_);
            seen_root_ = true;
            return kStart;
        }
    }

    // next() returns element tokens only, so this is its first token.
    bool next_start_element() { return next() == kStart; }

    void skip_current_element() {
        int depth = 1;
        while (depth) {
            const Token t = next();
            if (t == kDone || t == kError) return;
            if (t == kEnd) --depth;
            else ++depth;
        }
    }

    const std::string& name() const { return name_; }
    // The attribute's value, empty when absent (as the reference's lookups).
    std::string attr(const char* key) const {
        for (const auto& a : attrs_)
            if (a.first == key) return a.second;
        return std::string();
    }
    bool failed() const { return failed_; }
    const std::string& error() const { return err_; }

private:
    Token fail(const std::string& m) {
        if (!failed_) {
            failed_ = true;
            err_ = "XML error at byte " + std::to_string(p_) + ": " + m;
        }
        return kError;
    }
    bool skip_past(const char* tok) {
        const size_t q = s_.find(tok, p_);
        if (q == std::string::npos) return false;
        p_ = q + std::strlen(tok);
        return true;
    }
    bool skip_ws() {
        const size_t p0 = p_;
        while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\r' || s_[p_] == '\n')) ++p_;
        return p_ != p0;
    }
    std::string read_name() {
        const size_t p0 = p_;
        while (p_ < s_.size()) {
            const unsigned char c = (unsigned char)s_[p_];
            if (std::isalnum(c) || c == '_' || c == '-' || c == '.' || c == ':' || c >= 0x80) ++p_;
            else break;
        }
        return s_.substr(p0, p_ - p0);
    }
    static void put_utf8(uint32_t cp, std::string& out) {
        if (cp < 0x80) {
            out += (char)cp;
        } else if (cp < 0x800) {
            out += (char)(0xC0 | (cp >> 6));
            out += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += (char)(0xE0 | (cp >> 12));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        } else {
            out += (char)(0xF0 | (cp >> 18));
            out += (char)(0x80 | ((cp >> 12) & 0x3F));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        }
    }
    static bool decode(const std::string& in, std::string& out) {
        out.clear();
        for (size_t i = 0; i < in.size(); ++i) {
            if (in[i] != '&') {
                out += in[i];
                continue;
            }
            const size_t semi = in.find(';', i);
            if (semi == std::string::npos) return false;
            const std::string e = in.substr(i + 1, semi - i - 1);
            if (e == "lt") out += '<';
            else if (e == "gt") out += '>';
            else if (e == "amp") out += '&';
            else if (e == "quot") out += '"';
            else if (e == "apos") out += '\'';
            else if (e.size() > 1 && e[0] == '#') {
                const bool hex = e[1] == 'x' || e[1] == 'X';
                const std::string digits = e.substr(hex ? 2 : 1);
                if (digits.empty()) return false;
                char* end = nullptr;
                const unsigned long cp = std::strtoul(digits.c_str(), &end, hex ? 16 : 10);
                if (*end || cp == 0 || cp > 0x10FFFF) return false;
                put_utf8((uint32_t)cp, out);
            } else {
                return false;
            }
            i = semi;
        }
        return true;
    }

    std::string s_;
    size_t p_ = 0;
    std::string name_;
    std::vector<std::pair<std::string, std::string>> attrs_;
    std::vector<std::string> open_;
    bool pending_end_ = false;
    bool seen_root_ = false;
    bool failed_ = false;
    std::string err_;
};

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

// The attribute conversions of the reference: 0 when the text is not a
// number (or is absent).
int to_int(const std::string& s) {
    const std::string t = trim(s);
    if (t.empty()) return 0;
    errno = 0;
    char* end = nullptr;
    const long v = std::strtol(t.c_str(), &end, 10);
    if (*end || errno == ERANGE || v < INT32_MIN || v > INT32_MAX) return 0;
    return (int)v;
}

float to_float(const std::string& s) {
    const std::string t = trim(s);
    if (t.empty()) return 0.0f;
    char* end = nullptr;
    const float v = std::strtof(t.c_str(), &end);
    if (*end) return 0.0f;
    return v;
}

// DataSetReader::GetFilePath: the text before the last path separator; "."
// for a bare file name (where the reference would form "/voxels_<d>.gvb").
std::string dir_of(const std::string& path) {
    const size_t slash = path.find_last_of("/\\");
    if (slash == std::string::npos) return ".";
    return path.substr(0, slash);
}

bool read_text(const std::string& path, std::string& out, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

constexpr int kMaxLevels = 11;  // node encoding and walker path: levels 0..10

struct GvxLoader {
    XmlStream& xs;
    GvxFile& f;
    std::vector<std::vector<int32_t>> brick_nodes;  // per level: node of each brick index
    int max_level = 0;
    std::string err;

    // LoadOctTreeNode (GigaVoxelsReader.cpp:277-371) for the node record `cur`
    // whose start element was just read.
    bool load_node(size_t cur, int level, uint32_t parent) {
        if (to_int(xs.attr("Depth")) != level) {
            err = "Node Depth attribute " + xs.attr("Depth") + " does not match its depth " + std::to_string(level);
            return false;
        }
        GvxNode& n = f.nodes[cur];
        n.level = (int8_t)level;
        n.parent = parent;
        n.mip[0] = to_int(xs.attr("MipMapX"));
        n.mip[1] = to_int(xs.attr("MipMapY"));
        n.mip[2] = to_int(xs.attr("MipMapZ"));
        const std::string type = xs.attr("Type");
        if (type == "CONST" || type == "LEAF-CONST") {
            n.type = type == "CONST" ? kGvxConst : kGvxLeafConst;
            const uint32_t r = gvx_color_byte(to_float(xs.attr("ColorR")));
            const uint32_t g = gvx_color_byte(to_float(xs.attr("ColorG")));
            const uint32_t b = gvx_color_byte(to_float(xs.attr("ColorB")));
            const uint32_t a = gvx_color_byte(to_float(xs.attr("ColorA")));
            n.color = r | (g << 8) | (b << 16) | (a << 24);
        } else {
            n.type = kGvxNonConst;
            const int b = to_int(xs.attr("Brick"));
            if (b < 0) {
                err = "negative Brick index at depth " + std::to_string(level);
                return false;
            }
            // brick indices of a level are 0..n-1 for its n non-constant
            // nodes, and every node takes at least one "<Node" of the text:
            // a larger index can only be a corrupt file (and would size the
            // index list by it)
            if ((size_t)b >= xs.size() / 5 + 1) {
                err = "Brick index " + std::to_string(b) + " at depth " + std::to_string(level) +
                      " exceeds the number of nodes the file can hold";
                return false;
            }
            n.brick = b;
            std::vector<int32_t>& list = brick_nodes[(size_t)level];
            if ((size_t)b >= list.size()) list.resize((size_t)b + 1, -1);
            if (list[(size_t)b] >= 0) {
                err = "Brick index " + std::to_string(b) + " used twice at depth " + std::to_string(level);
                return false;
            }
            list[(size_t)b] = (int32_t)cur;
        }
        if (level == max_level || n.type == kGvxLeafConst) {
            xs.skip_current_element();
            if (xs.failed()) {
                err = xs.error();
                return false;
            }
            return true;
        }
        // allocateChildNodeBlock, then the next 8 start elements are the children
        const size_t block = f.nodes.size() / 8;
        f.nodes[cur].child_block = (int32_t)block;
        f.nodes.resize(f.nodes.size() + 8);
        for (int i = 0; i < 8; ++i) {
            XmlStream::Token t;
            do {
                t = xs.next();
            } while (t == XmlStream::kEnd);
            if (t != XmlStream::kStart) {
                err = xs.failed() ? xs.error() : "a Node at depth " + std::to_string(level) + " has fewer than 8 children";
                return false;
            }
            if (xs.name() != "Node") {
                err = "invalid element <" + xs.name() + "> where a child Node was expected";
                return false;
            }
            if (!load_node(block * 8 + (size_t)i, level + 1, (uint32_t)cur)) return false;
        }
        return true;
    }
};

template <class T>
bool read_pod(std::istream& in, T& v) {
    in.read((char*)&v, sizeof(T));
    return (size_t)in.gcount() == sizeof(T);
}

// LoadBinaryBricks (GigaVoxelsReader.cpp:106-221) for one level.
int load_bricks(const std::string& path, const std::vector<int32_t>& nodes, bool load_normals,
                 std::vector<GvxBrick>& out, std::string& err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        err = "cannot open " + path;
        return VV_ERR_IO;
    }
    int32_t compressed = 0;
    if (!read_pod(in, compressed)) {
        err = path + ": truncated header";
        return VV_ERR_IO;
    }
    out.clear();
    for (size_t i = 0; i < nodes.size() && nodes[i] >= 0; ++i) {
        uint64_t dims[3];
        uint32_t border[3];
        for (int a = 0; a < 3; ++a)
            if (!read_pod(in, dims[a])) {
                err = path + ": truncated brick " + std::to_string(i);
                return VV_ERR_IO;
            }
        for (int a = 0; a < 3; ++a)
            if (!read_pod(in, border[a])) {
                err = path + ": truncated brick " + std::to_string(i);
                return VV_ERR_IO;
            }
        GvxBrick b;
        for (int a = 0; a < 3; ++a) {
            // the 10^3 slot holds the stored texels from its origin; the node's
            // 8^3 voxels start at the border
            if (dims[a] < 1 || dims[a] > 10 || border[a] > 2) {
                err = path + ": brick " + std::to_string(i) + " has dims " + std::to_string(dims[a]) +
                      " / border " + std::to_string(border[a]) + " outside a 10^3 slot";
                return VV_ERR_ARG;
            }
            b.dims[a] = (uint8_t)dims[a];
            b.border[a] = (uint8_t)border[a];
        }
        const size_t count = (size_t)dims[0] * dims[1] * dims[2];
        for (int part = 0; part < 2; ++part) {
            const char* what = part == 0 ? "colors" : "gradients";
            int32_t c = 0;
            uint32_t size = 0;
            if (!read_pod(in, c) || !read_pod(in, size)) {
                err = path + ": truncated brick " + std::to_string(i);
                return VV_ERR_IO;
            }
            if (c != compressed) {
                err = path + ": compression mismatch found in brick file (" + what + ")";
                return VV_ERR_IO;
            }
            if (size == 0) {
                err = path + ": size of " + what + " data is zero";
                return VV_ERR_IO;
            }
            if (compressed) {
                err = path + ": DXT-compressed bricks are not supported";
                return VV_ERR_ARG;
            }
            const size_t want = count * (part == 0 ? 4 : 3);
            if (part == 1 && !load_normals) {
                in.seekg(size, std::ios::cur);
                if (!in) {
                    err = path + ": truncated brick " + std::to_string(i);
                    return VV_ERR_IO;
                }
                continue;
            }
            if (size != want) {
                err = path + ": brick " + std::to_string(i) + " " + what + " size " + std::to_string(size) +
                      " != " + std::to_string(want);
                return VV_ERR_IO;
            }
            std::vector<uint8_t>& dst = part == 0 ? b.colors : b.normals;
            dst.resize(size);
            in.read((char*)dst.data(), size);
            if ((size_t)in.gcount() != size) {
                err = path + ": tried to read " + std::to_string(size) + " " + what + " bytes, but read " +
                      std::to_string(in.gcount());
                return VV_ERR_IO;
            }
        }
        out.push_back(std::move(b));
    }
    if (in.peek() != std::char_traits<char>::eof()) {
        err = path + ": data after the last brick";
        return VV_ERR_IO;
    }
    return VV_OK;
}

}  // namespace

uint32_t gvx_color_byte(float value) {
    const float v = value * 255.0f;
    if (!(v > 0.0f)) return 0u;  // also NaN
    if (v >= 255.0f) return 255u;
    return (uint32_t)v;          // truncation, as the cast to unsigned char
}

float gvx_color_value(uint32_t v) {
    float f = (float)((double)v / 255.0);
    while (gvx_color_byte(f) < v) f = std::nextafter(f, 2.0f);
    while (v < 255u && gvx_color_byte(f) > v) f = std::nextafter(f, -1.0f);
    return f;
}

int read_gvx(const std::string& path, bool load_normals, GvxFile& out, std::string& err) {
    out = GvxFile();
    std::string text;
    if (!read_text(path, text, err)) return VV_ERR_IO;
    XmlStream xs(std::move(text));
    GvxLoader ld{xs, out, {}, 0, {}};
    bool have_header = false, have_tree = false;
    // LoadGVX (GigaVoxelsReader.cpp:373-514)
    while (xs.next_start_element()) {
        if (xs.name() == "GigaVoxelsOctTree") {
            if (have_header) {
                err = "more than one GigaVoxelsOctTree element";
                return VV_ERR_IO;
            }
            have_header = true;
            GvxHeader& h = out.h;
            const char* o[3] = {"X", "Y", "Z"};
            const char* d[3] = {"DeltaX", "DeltaY", "DeltaZ"};
            const char* v[3] = {"VolumeXSize", "VolumeYSize", "VolumeZSize"};
            const char* b[3] = {"BrickXSize", "BrickYSize", "BrickZSize"};
            for (int a = 0; a < 3; ++a) {
                h.origin[a] = to_float(xs.attr(o[a]));
                h.delta[a] = to_float(xs.attr(d[a]));
                h.volume_size[a] = to_int(xs.attr(v[a]));
                h.brick_size[a] = to_int(xs.attr(b[a]));
            }
            h.binary = xs.attr("Binary") == "YES";
            h.compressed = xs.attr("Compressed") == "YES";
            h.max_depth = to_int(xs.attr("MaxDepth"));
            if (h.max_depth < 1 || h.max_depth > kMaxLevels) {
                err = "MaxDepth " + std::to_string(h.max_depth) + " outside 1.." + std::to_string(kMaxLevels);
                return h.max_depth < 1 ? VV_ERR_IO : VV_ERR_ARG;
            }
            if (h.brick_size[0] != 8 || h.brick_size[1] != 8 || h.brick_size[2] != 8) {
                err = "brick size " + std::to_string(h.brick_size[0]) + "x" + std::to_string(h.brick_size[1]) + "x" +
                      std::to_string(h.brick_size[2]) + " is not supported (8x8x8 only)";
                return VV_ERR_ARG;
            }
        } else if (have_header && xs.name() == "Node") {
            if (have_tree) {
                err = "more than one root Node";
                return VV_ERR_IO;
            }
            have_tree = true;
            ld.max_level = out.h.max_depth - 1;
            ld.brick_nodes.assign((size_t)out.h.max_depth, {});
            out.nodes.assign(8, GvxNode());  // the root block: the root is record 0
            if (!ld.load_node(0, 0, 0xFFFFFFFFu)) {
                err = ld.err;
                return VV_ERR_IO;
            }
            xs.skip_current_element();
            out.bricks.assign((size_t)out.h.max_depth, {});
            const std::string dir = dir_of(path);
            for (size_t lv = 0; lv < ld.brick_nodes.size(); ++lv) {
                const std::vector<int32_t>& list = ld.brick_nodes[lv];
                if (list.empty()) continue;
                if (!out.h.binary) {
                    err = "binary bricks are the only supported format";
                    return VV_ERR_IO;
                }
                if (out.h.compressed) {
                    err = "DXT-compressed bricks are not supported";
                    return VV_ERR_ARG;
                }
                const std::string bp = dir + "/voxels_" + std::to_string(lv) + ".gvb";
                const int rc = load_bricks(bp, list, load_normals, out.bricks[lv], err);
                if (rc) return rc;
                // a node whose index lies after a gap would have no brick
                if (out.bricks[lv].size() != list.size()) {
                    err = bp + ": Brick index " + std::to_string(out.bricks[lv].size()) + " missing at depth " +
                          std::to_string(lv);
                    return VV_ERR_IO;
                }
            }
        }
    }
    if (xs.failed()) {
        err = xs.error();
        return VV_ERR_IO;
    }
    if (!have_tree) {
        err = have_header ? "no Node element" : "no GigaVoxelsOctTree element";
        return VV_ERR_IO;
    }
    return VV_OK;
}

namespace {

std::string fmt_float(float v) {
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%.9g", (double)v);
    return buf;
}

// WriteOctTreeNode (Voxelizer.cu:2840-2995): one Node element and, unless it
// is a leaf, its 8 children.
void write_node(std::ostream& o, const GvxFile& f, size_t n) {
    const GvxNode& nd = f.nodes[n];
    for (int i = 0; i <= nd.level; ++i) o << "    ";
    o << "<Node MipMapX=\"" << nd.mip[0] << "\" MipMapY=\"" << nd.mip[1] << "\" MipMapZ=\"" << nd.mip[2] << "\" ";
    if (nd.type == kGvxNonConst) {
        o << "Type=\"NON-CONST\" Brick=\"" << nd.brick << "\" ";
    } else {
        o << "Type=\"" << (nd.type == kGvxConst ? "CONST" : "LEAF-CONST") << "\" ";
        const char* ch[4] = {"ColorR", "ColorG", "ColorB", "ColorA"};
        for (int c = 0; c < 4; ++c) o << ch[c] << "=\"" << fmt_float(gvx_color_value((nd.color >> (8 * c)) & 255u)) << "\" ";
    }
    o << "Depth=\"" << (int)nd.level << "\"";
    if (nd.child_block >= 0) {
        o << ">\n";
        for (int c = 0; c < 8; ++c) write_node(o, f, (size_t)nd.child_block * 8 + (size_t)c);
        for (int i = 0; i <= nd.level; ++i) o << "    ";
        o << "</Node>\n";
    } else {
        o << " />\n";
    }
}

}  // namespace

bool write_gvx(const std::string& dir, const GvxFile& f, std::string& err) {
    std::vector<size_t> per_level(f.bricks.size());
    for (size_t lv = 0; lv < f.bricks.size(); ++lv) per_level[lv] = f.bricks[lv].size();
    return write_gvx(dir, f, per_level, [&](size_t lv, size_t i, GvxBrick& b) { b = f.bricks[lv][i]; }, err);
}

bool write_gvx(const std::string& dir, const GvxFile& f, const std::vector<size_t>& bricks_per_level,
               const GvxBrickSource& source, std::string& err) {
    const GvxHeader& h = f.h;
    if (f.nodes.empty() || f.nodes[0].level != 0) {
        err = "the tree has no root";
        return false;
    }
    {
        std::ofstream o(dir + "/tree.gvx", std::ios::binary);
        if (!o) {
            err = "cannot create " + dir + "/tree.gvx";
            return false;
        }
        // writeOctTree (Voxelizer.cu:2998-3058)
        o << "<GigaVoxelsOctTree MaxDepth=\"" << h.max_depth << "\" X=\"" << fmt_float(h.origin[0]) << "\" Y=\""
          << fmt_float(h.origin[1]) << "\" Z=\"" << fmt_float(h.origin[2]) << "\" DeltaX=\"" << fmt_float(h.delta[0])
          << "\" DeltaY=\"" << fmt_float(h.delta[1]) << "\" DeltaZ=\"" << fmt_float(h.delta[2])
          << "\" VolumeXSize=\"" << h.volume_size[0] << "\" VolumeYSize=\"" << h.volume_size[1]
          << "\" VolumeZSize=\"" << h.volume_size[2] << "\" BrickXSize=\"" << h.brick_size[0] << "\" BrickYSize=\""
          << h.brick_size[1] << "\" BrickZSize=\"" << h.brick_size[2] << "\" Binary=\"" << (h.binary ? "YES" : "NO")
          << "\" Compressed=\"" << (h.compressed ? "YES" : "NO") << "\" >\n";
        write_node(o, f, 0);
        o << "</GigaVoxelsOctTree>\n";
        if (!o) {
            err = "write failed: " + dir + "/tree.gvx";
            return false;
        }
    }
    GvxBrick b;
    for (size_t lv = 0; lv < bricks_per_level.size(); ++lv) {
        if (bricks_per_level[lv] == 0) continue;
        const std::string bp = dir + "/voxels_" + std::to_string(lv) + ".gvb";
        std::ofstream o(bp, std::ios::binary);
        if (!o) {
            err = "cannot create " + bp;
            return false;
        }
        // startBricksFile (VoxelBrickWriter.cu:71-110), WriteBinaryBrick (:726-818)
        const int32_t compressed = 0;
        o.write((const char*)&compressed, 4);
        for (size_t i = 0; i < bricks_per_level[lv]; ++i) {
            source(lv, i, b);
            const size_t count = (size_t)b.dims[0] * b.dims[1] * b.dims[2];
            for (int a = 0; a < 3; ++a) {
                const uint64_t d = b.dims[a];
                o.write((const char*)&d, 8);
            }
            for (int a = 0; a < 3; ++a) {
                const uint32_t bd = b.border[a];
                o.write((const char*)&bd, 4);
            }
            if (b.colors.size() != count * 4 || (!b.normals.empty() && b.normals.size() != count * 3)) {
                err = "brick payload does not match its dims";
                return false;
            }
            std::vector<uint8_t> nrm;
            const std::vector<uint8_t>* np = &b.normals;
            if (b.normals.empty()) {  // a tree without gradients: the zero vector, unsigned
                nrm.assign(count * 3, 128);
                np = &nrm;
            }
            uint32_t size = (uint32_t)b.colors.size();
            o.write((const char*)&compressed, 4);
            o.write((const char*)&size, 4);
            o.write((const char*)b.colors.data(), size);
            size = (uint32_t)np->size();
            o.write((const char*)&compressed, 4);
            o.write((const char*)&size, 4);
            o.write((const char*)np->data(), size);
        }
        if (!o) {
            err = "write failed: " + bp;
            return false;
        }
    }
    return true;
}

namespace {

// BoundingSphere::expandBy (VoxVizCore/BoundingVolumes.cpp:48-107).
void expand_sphere(float c[3], double& r, const float cc[3], double rr) {
    if (!(rr > 0.0)) return;
    if (!(r > 0.0)) {
        for (int a = 0; a < 3; ++a) c[a] = cc[a];
        r = rr;
        return;
    }
    const double dx = (double)c[0] - cc[0], dy = (double)c[1] - cc[1], dz = (double)c[2] - cc[2];
    const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (d + rr <= r) return;
    if (d + r <= rr) {
        for (int a = 0; a < 3; ++a) c[a] = cc[a];
        r = rr;
        return;
    }
    const double nr = (r + d + rr) * 0.5;
    const double ratio = (nr - r) / d;
    for (int a = 0; a < 3; ++a) c[a] = (float)((double)c[a] + ((double)cc[a] - (double)c[a]) * ratio);
    r = nr;
}

}  // namespace

int read_gvp(const std::string& path, GvpFile& out, std::string& err) {
    out = GvpFile();
    std::string text;
    if (!read_text(path, text, err)) return VV_ERR_IO;
    XmlStream xs(std::move(text));
    bool have_root = false;
    const std::string dir = dir_of(path);
    // LoadGVP (GigaVoxelsReader.cpp:35-101)
    while (xs.next_start_element()) {
        if (xs.name() == "OctTrees") {
            have_root = true;
            out.compressed = xs.attr("Compressed") == "YES";
            out.brick_size[0] = to_int(xs.attr("BrickXSize"));
            out.brick_size[1] = to_int(xs.attr("BrickYSize"));
            out.brick_size[2] = to_int(xs.attr("BrickZSize"));
        } else if (have_root && xs.name() == "OctTree") {
            GvpTile t;
            t.center[0] = to_float(xs.attr("CenterX"));
            t.center[1] = to_float(xs.attr("CenterY"));
            t.center[2] = to_float(xs.attr("CenterZ"));
            t.radius = to_float(xs.attr("Radius"));
            t.size_meters[0] = to_float(xs.attr("SizeXMeters"));
            t.size_meters[1] = to_float(xs.attr("SizeYMeters"));
            t.size_meters[2] = to_float(xs.attr("SizeZMeters"));
            t.tree_file = dir + "/" + xs.attr("TreeFile");
            expand_sphere(out.sphere_center, out.sphere_radius, t.center, (double)t.radius);
            out.tiles.push_back(std::move(t));
            xs.skip_current_element();
        }
    }
    if (xs.failed()) {
        err = xs.error();
        return VV_ERR_IO;
    }
    if (!have_root) {
        err = "no OctTrees element";
        return VV_ERR_IO;
    }
    return VV_OK;
}

bool write_gvp(const std::string& path, const GvpFile& f, std::string& err) {
    std::ofstream o(path, std::ios::binary);
    if (!o) {
        err = "cannot create " + path;
        return false;
    }
    // the root file of the voxelizer (main.cu:4420-4480)
    o << "<OctTrees Compressed='" << (f.compressed ? "YES" : "NO") << "' BrickXSize='" << f.brick_size[0]
      << "' BrickYSize='" << f.brick_size[1] << "' BrickZSize='" << f.brick_size[2] << "' >\n";
    for (const GvpTile& t : f.tiles) {
        std::string file;  // relative to the .gvp's directory
        for (char c : t.tree_file) {
            if (c == '&') file += "&amp;";
            else if (c == '<') file += "&lt;";
            else if (c == '"') file += "&quot;";
            else file += c;
        }
        o << "    <OctTree CenterX=\"" << fmt_float(t.center[0]) << "\" CenterY=\"" << fmt_float(t.center[1])
          << "\" CenterZ=\"" << fmt_float(t.center[2]) << "\" Radius=\"" << fmt_float(t.radius)
          << "\" SizeXMeters=\"" << fmt_float(t.size_meters[0]) << "\" SizeYMeters=\"" << fmt_float(t.size_meters[1])
          << "\" SizeZMeters=\"" << fmt_float(t.size_meters[2]) << "\" TreeFile=\"" << file << "\" />\n";
    }
    o << "</OctTrees>\n";
    if (!o) {
        err = "write failed: " + path;
        return false;
    }
    return true;
}

}  // namespace vv
