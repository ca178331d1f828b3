// .dsml scene loader: the reference's input format (src/parser.cpp:49-377,
// src/DEMSimulation.cpp:45-60) and its scene construction (PrepareSim,
// src/main.cu:54-369, with the block generators createRectanglesD and
// createTrianglesD, particles_kernel.cuh:43-111), host only.
//
// A .dsml file is a small XML document.  The reader below handles what such
// files contain (declaration, comments, elements, attributes, text) and, like
// the reference's, looks only at the element children of each node.  The
// rules of the scene follow the reference: which tags are required, their
// defaults and error texts, type ids, particle order (single particles, then
// rectangles, then triangles), the followed list (single particles with
// follow="true", then the <follow> ids) and the grid rule of main.cu:218-236.
//
// The rectangle generator jitters each lattice point by (N(0,1) - 0.5) / 100
// of the lattice spacing, as the reference does with cuRAND.  The reference
// seeds cuRAND with time(NULL); here the seed is an argument and each deviate
// comes from a counter-based SplitMix64 hash and a Box-Muller transform, so a
// scene is reproducible.  DEM_DSML_NO_JITTER uses a deviate of 0.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/demso_b200.h"

int dem_record_error(int code, const char* msg);  // dem_api.cu

namespace {

template <typename... A>
int record(int code, const char* fmt, A... args) {
    char msg[512];
    snprintf(msg, sizeof(msg), fmt, args...);
    return dem_record_error(code, msg);
}

// ---------------------------------------------------------------- XML reader
struct Node {
    std::string name, text;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<Node> kids;  // element children only
    const Node* child(const char* n) const {
        for (const Node& k : kids)
            if (k.name == n) return &k;
        return nullptr;
    }
    const char* attr(const char* n) const {
        for (const auto& a : attrs)
            if (a.first == n) return a.second.c_str();
        return nullptr;
    }
};

struct XmlError {
    std::string msg;
};

class Reader {
  public:
    Reader(const char* s, size_t n) : p_(s), e_(s + n) {}
    Node document() {
        Node root;
        root.name = "#document";
        content(root, true);
        return root;
    }

  private:
    const char *p_, *e_;
    [[noreturn]] void fail(const char* what) { throw XmlError{what}; }
    bool starts(const char* t) const {
        const size_t n = strlen(t);
        return (size_t)(e_ - p_) >= n && memcmp(p_, t, n) == 0;
    }
    void skip_to(const char* t) {
        const size_t n = strlen(t);
        while (p_ < e_ && !starts(t)) ++p_;
        if (p_ >= e_) fail("unterminated markup");
        p_ += n;
    }
    static bool space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }
    static bool name_char(char c) {
        return !space(c) && c != '>' && c != '/' && c != '=' && c != '<' && c != '"' && c != '\'';
    }
    static std::string decode(const char* a, const char* b) {
        static const struct {
            const char* ent;
            char c;
        } tab[] = {{"&lt;", '<'}, {"&gt;", '>'}, {"&amp;", '&'}, {"&quot;", '"'}, {"&apos;", '\''}};
        std::string out;
        for (const char* q = a; q < b; ++q) {
            bool done = false;
            if (*q == '&') {
                for (const auto& t : tab) {
                    const size_t n = strlen(t.ent);
                    if ((size_t)(b - q) >= n && memcmp(q, t.ent, n) == 0) {
                        out += t.c;
                        q += n - 1;
                        done = true;
                        break;
                    }
                }
            }
            if (!done) out += *q;
        }
        return out;
    }
    // children and text of `parent`, up to its end tag (or the end of input)
    void content(Node& parent, bool top) {
        while (p_ < e_) {
            if (starts("<!--")) {
                skip_to("-->");
            } else if (starts("<?")) {
                skip_to("?>");
            } else if (starts("<!")) {
                skip_to(">");
            } else if (starts("</")) {
                if (top) fail("unexpected end tag");
                p_ += 2;
                const char* a = p_;
                while (p_ < e_ && name_char(*p_)) ++p_;
                if (std::string(a, p_) != parent.name) fail("mismatched end tag");
                skip_to(">");
                return;
            } else if (*p_ == '<') {
                parent.kids.emplace_back();
                element(parent.kids.back());
            } else {
                const char* a = p_;
                while (p_ < e_ && *p_ != '<') ++p_;
                bool blank = true;
                for (const char* q = a; q < p_; ++q) blank = blank && space(*q);
                if (!blank && parent.text.empty()) parent.text = decode(a, p_);
            }
        }
        if (!top) fail("unterminated element");
    }
    void element(Node& n) {
        ++p_;  // '<'
        const char* a = p_;
        while (p_ < e_ && name_char(*p_)) ++p_;
        n.name.assign(a, p_);
        if (n.name.empty()) fail("empty element name");
        for (;;) {
            while (p_ < e_ && space(*p_)) ++p_;
            if (p_ >= e_) fail("unterminated tag");
            if (starts("/>")) {
                p_ += 2;
                return;
            }
            if (*p_ == '>') {
                ++p_;
                content(n, false);
                return;
            }
            const char* k = p_;
            while (p_ < e_ && name_char(*p_)) ++p_;
            std::string key(k, p_);
            while (p_ < e_ && space(*p_)) ++p_;
            if (p_ >= e_ || *p_ != '=') fail("attribute without value");
            ++p_;
            while (p_ < e_ && space(*p_)) ++p_;
            if (p_ >= e_ || (*p_ != '"' && *p_ != '\'')) fail("unquoted attribute value");
            const char q = *p_++;
            const char* v = p_;
            while (p_ < e_ && *p_ != q) ++p_;
            if (p_ >= e_) fail("unterminated attribute value");
            n.attrs.emplace_back(key, decode(v, p_));
            ++p_;
        }
    }
};

// ------------------------------------------------------------ scene content
struct PType {
    std::string id, name;
    float mass = 0, radius = 0, kn = 0, kt = 0, cn = 0, eb = 0, mu = 0, at = 0;
    float color[3] = {255, 255, 255};
};
struct Rect {
    float sx, sy, ex, ey;
    uint32_t nx, ny;
    std::vector<int> types;
};
struct Tri {
    float px, py, width;
    uint32_t num;
    std::vector<int> types;
};
struct Single {
    float px, py, vx, vy, theta, omega;
    int type;
};

struct Scene {
    float timeStep = -1, simDuration = -1;
    uint32_t imageHeight = 800;
    std::vector<int> paramFollow;
    float dim[2] = {0, 0}, grav[2] = {0, 0}, knWall = 0, ktWall = 0;
    std::vector<PType> types;
    std::vector<Rect> rects;
    std::vector<Tri> tris;
    std::vector<Single> singles;
    std::vector<int> singleFollow;
    int controlled = -1;
    // generated state
    std::vector<float> pos, vel, theta, omega, radius, mass;
    std::vector<uint32_t> id, type;
};

struct SemErr {
    std::string msg;
};

float num(const Node& n) { return (float)atof(n.text.c_str()); }

// parser.cpp:352-362: the <x> and <y> children, 0 when absent
void vec2(const Node& n, float& x, float& y) {
    x = y = 0.0f;
    for (const Node& k : n.kids) {
        if (k.name == "x") x = num(k);
        else if (k.name == "y") y = num(k);
    }
}

// DEMSimulation.cpp:37-42
int type_index(const Scene& s, const std::string& id) {
    for (size_t i = 0; i < s.types.size(); ++i)
        if (s.types[i].id == id) return (int)i;
    throw SemErr{"Nonexistant particle id: '" + id + "'"};
}

// parser.cpp:364-377: fields split on ',' with spaces kept
std::vector<int> type_list(const Scene& s, const char* csv) {
    std::vector<int> out;
    const std::string line(csv);
    std::string cur;
    for (size_t i = 0; i <= line.size(); ++i) {
        if (i == line.size() || line[i] == ',') {
            out.push_back(type_index(s, cur));
            cur.clear();
        } else {
            cur += line[i];
        }
    }
    return out;
}

float hex_byte(const std::string& h) { return (float)strtol(h.c_str(), nullptr, 16); }

void load(Scene& s, const Node& doc) {
    const Node* root = doc.child("simulation");
    if (!root) throw SemErr{"<simulation> not found"};
    // parser.cpp:49-76
    const Node* par = root->child("parameters");
    if (!par) throw SemErr{"<parameters> not found"};
    for (const Node& k : par->kids) {
        if (k.name == "timestep") s.timeStep = num(k);
        else if (k.name == "simduration") s.simDuration = num(k);
        else if (k.name == "imageheight") s.imageHeight = (uint32_t)atoi(k.text.c_str());
        else if (k.name == "follow") s.paramFollow.push_back(atoi(k.text.c_str()));
    }
    if (s.timeStep == -1) throw SemErr{"Simulation timestep not specified"};
    // parser.cpp:77-95
    const Node* env = root->child("environment");
    if (!env) throw SemErr{"<environment> not found"};
    for (const Node& k : env->kids) {
        if (k.name == "dimensions") {
            vec2(k, s.dim[0], s.dim[1]);
        } else if (k.name == "gravity") {
            vec2(k, s.grav[0], s.grav[1]);
        } else if (k.name == "stiffness") {
            const char* d = k.attr("dir");
            if (!d) throw SemErr{"Stiffness direction not specified"};
            if (std::string(d) == "normal") s.knWall = num(k);
            else if (std::string(d) == "shear") s.ktWall = num(k);
            else throw SemErr{"Unrecognized stiffness direction"};
        }
    }
    // parser.cpp:97-167
    if (const Node* pr = root->child("properties")) {
        for (const Node& k : pr->kids) {
            if (k.name != "particletype") continue;
            PType t;
            if (const char* a = k.attr("id")) t.id = a;
            if (const char* a = k.attr("name")) t.name = a;
            if (const char* a = k.attr("color")) {
                const std::string c(a);
                t.color[0] = hex_byte(c.substr(0, 2));
                t.color[1] = hex_byte(c.size() > 2 ? c.substr(2, 2) : "");
                t.color[2] = hex_byte(c.size() > 4 ? c.substr(4, 2) : "");
            }
            for (const Node& q : k.kids) {
                if (q.name == "mass") {
                    t.mass = num(q);
                } else if (q.name == "radius") {
                    t.radius = num(q);
                } else if (q.name == "stiffness") {
                    const char* d = q.attr("dir");
                    if (!d) throw SemErr{"Stiffness direction not specified"};
                    if (std::string(d) == "normal") t.kn = num(q);
                    else if (std::string(d) == "shear") t.kt = num(q);
                    else throw SemErr{"Unrecognized stiffness direction"};
                } else if (q.name == "damping") {
                    const char* d = q.attr("type");
                    if (d) {
                        if (std::string(d) == "boundary") t.eb = num(q);
                        else throw SemErr{"Unrecognized damping type"};
                    } else {
                        t.cn = num(q);
                    }
                } else if (q.name == "friction") {
                    t.mu = num(q);
                } else if (q.name == "attraction") {
                    t.at = num(q);
                } else {
                    throw SemErr{"Unrecognized tag inside <particletype>"};
                }
            }
            s.types.push_back(t);
        }
    }
    // parser.cpp:169-350
    const Node* pa = root->child("particles");
    if (!pa) throw SemErr{"<particles> not found"};
    if (s.types.empty()) throw SemErr{"No particle types defined, aborting."};
    for (const Node& k : pa->kids) {
        if (k.name == "rectangle") {
            Rect r;
            const char* a = k.attr("particletype");
            r.types = a ? type_list(s, a) : std::vector<int>(1, 0);
            const Node* st = k.child("start");
            if (!st) throw SemErr{"<start> tag not found inside rectangle"};
            vec2(*st, r.sx, r.sy);
            const Node* en = k.child("end");
            if (!en) throw SemErr{"<end> tag not found inside rectangle"};
            vec2(*en, r.ex, r.ey);
            const Node* nm = k.child("num");
            if (!nm) throw SemErr{"<num> tag not found inside rectangle"};
            float fx, fy;
            vec2(*nm, fx, fy);
            r.nx = (uint32_t)fx;
            r.ny = (uint32_t)fy;
            s.rects.push_back(r);
        } else if (k.name == "triangle") {
            Tri t;
            const char* a = k.attr("particletype");
            t.types = a ? type_list(s, a) : std::vector<int>(1, 0);
            const Node* ps = k.child("pos");
            if (!ps) throw SemErr{"<pos> tag not found inside triangle"};
            vec2(*ps, t.px, t.py);
            const Node* w = k.child("width");
            if (!w) throw SemErr{"<width> tag not found inside triangle"};
            t.width = num(*w);
            const Node* nm = k.child("num");
            if (!nm) throw SemErr{"<num> tag not found inside triangle"};
            t.num = (uint32_t)atoi(nm->text.c_str());
            s.tris.push_back(t);
        } else if (k.name == "particle") {
            Single p;
            const char* a = k.attr("particletype");
            p.type = a ? type_index(s, a) : 0;
            const char* f = k.attr("follow");
            if (f && std::string(f) == "true") s.singleFollow.push_back((int)s.singles.size());
            const Node* ps = k.child("pos");
            if (!ps) throw SemErr{"Missing <pos> tag on particle definition"};
            vec2(*ps, p.px, p.py);
            p.vx = p.vy = 0.0f;
            if (const Node* v = k.child("vel")) vec2(*v, p.vx, p.vy);
            const Node* th = k.child("theta");
            p.theta = th ? num(*th) : 0.0f;
            const Node* om = k.child("omega");
            p.omega = om ? num(*om) : 0.0f;
            s.singles.push_back(p);
        } else if (k.name == "controlled") {
            // read only with USE_BIG_PARTICLE 1 (parser.cpp:325-347): reported,
            // never an error here
            const char* a = k.attr("particletype");
            s.controlled = 0;
            if (a) {
                s.controlled = -1;
                for (size_t i = 0; i < s.types.size(); ++i)
                    if (s.types[i].id == a) s.controlled = (int)i;
            }
        }
    }
}

// SplitMix64 (Steele, Lea and Flood, 2014) and a Box-Muller normal deviate
uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
float normal_deviate(uint64_t seed, uint64_t stream, uint64_t k) {
    const uint64_t a = splitmix(seed ^ splitmix(stream * 4 + k));
    const uint64_t b = splitmix(a);
    const double u1 = ((double)(a >> 11) + 1.0) * (1.0 / 9007199254740992.0);  // (0, 1]
    const double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);          // [0, 1)
    return (float)(std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
}

void generate(Scene& s, uint64_t seed, bool jitter) {
    auto add = [&](float x, float y, float vx, float vy, float th, float om, int t) {
        s.pos.push_back(x);
        s.pos.push_back(y);
        s.vel.push_back(vx);
        s.vel.push_back(vy);
        s.theta.push_back(th);
        s.omega.push_back(om);
        s.radius.push_back(s.types[t].radius);
        s.mass.push_back(s.types[t].mass);
        s.id.push_back((uint32_t)s.id.size());
        s.type.push_back((uint32_t)t);
    };
    // main.cu:249-267: single particles first
    for (const Single& p : s.singles) add(p.px, p.py, p.vx, p.vy, p.theta, p.omega, p.type);
    // main.cu:270-295 and particles_kernel.cuh:43-74 (createRectanglesD), in
    // file order; the float operations are the reference's
    for (size_t b = 0; b < s.rects.size(); ++b) {
        const Rect& r = s.rects[b];
        const float lx = r.ex - r.sx, ly = r.ey - r.sy;
        const uint32_t nt = (uint32_t)r.types.size();
        for (uint32_t y = 0; y < r.ny; ++y)
            for (uint32_t x = 0; x < r.nx; ++x) {
                const uint32_t particle = x + y * r.nx;
                const uint64_t stream = ((uint64_t)b << 32) | particle;
                const float n1 = jitter ? normal_deviate(seed, stream, 0) : 0.0f;
                const float n2 = jitter ? normal_deviate(seed, stream, 1) : 0.0f;
                const float px = r.sx + lx / (float)(r.nx - 1) * ((float)x + (n1 - 0.5f) / 100);
                const float py = r.sy + ly / (float)(r.ny - 1) * ((float)y + (n2 - 0.5f) / 100);
                add(px, py, 0.0f, 0.0f, 0.0f, 0.0f, r.types[(x + y) % nt]);
            }
    }
    // main.cu:298-325 and particles_kernel.cuh:76-111 (createTrianglesD): row
    // L of a triangle of N on its base holds N - L particles; the integer and
    // float operations (and their types) are the reference's
    for (const Tri& t : s.tris) {
        const uint32_t N = t.num;
        const uint32_t count = N * (N + 1) / 2;
        const float space = t.width / (float)(N - 1);
        const float height = (float)(space * std::sqrt(3.0) / 2);
        const uint32_t nt = (uint32_t)t.types.size();
        for (uint32_t index = 0; index < count; ++index) {
            const int L1 = (int)((1 + 2 * sqrtf((float)(N * N + N - 2 * (index + 1) + 1))) / 2);
            const int L = (int)(N - (uint32_t)L1);
            const int first = (int)(((uint32_t)L1 + N + N * N - (uint32_t)(L1 * L1)) / 2);
            const int C = (int)index - first + L1;
            const int A = (int)(N - 1);
            const float px = t.px + (float)(L + 2 * C - A) * space / 2;
            const float py = t.py + (float)L * height;
            add(px, py, 0.0f, 0.0f, 0.0f, 0.0f, t.types[(uint32_t)(C + L) % nt]);
        }
    }
}

// main.cu:218-236, with log2(x) = log(x)/log(2) in double (main.cu:38) and
// the float arithmetic of the reference; the y axis measures its cell with
// the box's x size, as the reference does
uint32_t grid_axis(float cells, float cellLen, float maxRadius) {
    const uint32_t grid = (uint32_t)cells;
    uint32_t temp = grid > 0 ? (uint32_t)(std::log((double)grid) / std::log(2.0)) : 0u;
    const uint32_t upd = 1u << temp;
    const float cell = cellLen / (float)upd;
    if (cell / 2.0f <= 1.2f * maxRadius) temp -= 1;
    else if (cell / 2.0f >= 3.0f * maxRadius) temp += 1;
    return 1u << temp;
}

}  // namespace

struct DemDsml {
    Scene s;
};

extern "C" int dem_dsml_parse(const char* text, size_t length, uint64_t seed, uint32_t flags,
                              DemDsml** out) {
    if (!text || !out) return record(DEM_ERR_INVALID_ARG, "%s", "dem_dsml_parse: NULL argument");
    *out = nullptr;
    DemDsml* d = new DemDsml();
    try {
        Reader r(text, length);
        const Node doc = r.document();
        load(d->s, doc);
    } catch (const XmlError& e) {
        delete d;
        return record(DEM_ERR_INVALID_ARG, "dsml: XML: %s", e.msg.c_str());
    } catch (const SemErr& e) {
        delete d;
        return record(DEM_ERR_INVALID_ARG, "Parsing Error: %s", e.msg.c_str());
    }
    if (d->s.types.size() > DEM_MAX_MATERIALS) {
        const size_t nt = d->s.types.size();
        delete d;
        return record(DEM_ERR_INVALID_ARG, "dsml: %zu particle types (at most %d)", nt,
                      DEM_MAX_MATERIALS);
    }
    generate(d->s, seed, !(flags & DEM_DSML_NO_JITTER));
    *out = d;
    return DEM_OK;
}

extern "C" int dem_dsml_load(const char* path, uint64_t seed, uint32_t flags, DemDsml** out) {
    if (!path || !out) return record(DEM_ERR_INVALID_ARG, "%s", "dem_dsml_load: NULL argument");
    FILE* f = fopen(path, "rb");
    if (!f) return record(DEM_ERR_INVALID_ARG, "dsml: cannot open %s", path);
    std::string text;
    char buf[65536];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    fclose(f);
    return dem_dsml_parse(text.data(), text.size(), seed, flags, out);
}

extern "C" void dem_dsml_free(DemDsml* d) { delete d; }

extern "C" int dem_dsml_info(const DemDsml* d, DemDsmlInfo* info) {
    if (!d || !info) return record(DEM_ERR_INVALID_ARG, "%s", "dem_dsml_info: NULL argument");
    const Scene& s = d->s;
    memset(info, 0, sizeof(*info));
    info->numParticles = (uint32_t)s.id.size();
    info->numTypes = (uint32_t)s.types.size();
    info->numFollowed = (uint32_t)(s.singleFollow.size() + s.paramFollow.size());
    info->imageHeight = s.imageHeight;
    info->numRectangles = (uint32_t)s.rects.size();
    info->numTriangles = (uint32_t)s.tris.size();
    info->numSingles = (uint32_t)s.singles.size();
    info->controlledType = s.controlled;
    info->timeStep = s.timeStep;
    info->simDuration = s.simDuration;
    return DEM_OK;
}

extern "C" int dem_dsml_system(const DemDsml* d, DemSystem* sys) {
    if (!d || !sys) return record(DEM_ERR_INVALID_ARG, "%s", "dem_dsml_system: NULL argument");
    const Scene& s = d->s;
    memset(sys, 0, sizeof(*sys));
    sys->numParticles = (uint32_t)s.id.size();
    sys->cubeDimension[0] = s.dim[0];
    sys->cubeDimension[1] = s.dim[1];
    sys->timeStep = s.timeStep;
    sys->gravity[0] = s.grav[0];
    sys->gravity[1] = s.grav[1];
    sys->boundaryNormalStiffness = s.knWall;
    sys->boundaryShearStiffness = s.ktWall;
    sys->numMaterials = (uint32_t)s.types.size();
    // main.cu:199-208: the largest radius over all particle types (the
    // control particle's type is skipped only with USE_BIG_PARTICLE 1; the
    // step here has no control particle)
    float maxRadius = 0.0f;
    for (size_t t = 0; t < s.types.size(); ++t) {
        const PType& p = s.types[t];
        sys->materials[t] = DemMaterial{p.kn, p.kt, p.cn, p.eb, p.mu, p.at};
        if (maxRadius < p.radius) maxRadius = p.radius;
    }
    sys->gridSize[0] = grid_axis(s.dim[0] / (4.0f * maxRadius), s.dim[0], maxRadius);
    sys->gridSize[1] = grid_axis(s.dim[1] / (4.0f * maxRadius), s.dim[0], maxRadius);
    return DEM_OK;
}

extern "C" int dem_dsml_state(const DemDsml* d, float* pos, float* vel, float* theta, float* omega,
                              float* radius, float* mass, uint32_t* id, uint32_t* type) {
    if (!d) return record(DEM_ERR_INVALID_ARG, "%s", "dem_dsml_state: NULL scene");
    const Scene& s = d->s;
    const size_t n = s.id.size();
    auto cp = [](void* dst, const void* src, size_t bytes) {
        if (dst && bytes) memcpy(dst, src, bytes);
    };
    cp(pos, s.pos.data(), 8 * n);
    cp(vel, s.vel.data(), 8 * n);
    cp(theta, s.theta.data(), 4 * n);
    cp(omega, s.omega.data(), 4 * n);
    cp(radius, s.radius.data(), 4 * n);
    cp(mass, s.mass.data(), 4 * n);
    cp(id, s.id.data(), 4 * n);
    cp(type, s.type.data(), 4 * n);
    return DEM_OK;
}

extern "C" int dem_dsml_followed(const DemDsml* d, uint32_t* ids) {
    if (!d || !ids) return record(DEM_ERR_INVALID_ARG, "%s", "dem_dsml_followed: NULL argument");
    size_t k = 0;
    for (int v : d->s.singleFollow) ids[k++] = (uint32_t)v;
    for (int v : d->s.paramFollow) ids[k++] = (uint32_t)v;
    return DEM_OK;
}

extern "C" int dem_dsml_type(const DemDsml* d, uint32_t t, DemDsmlType* out) {
    if (!d || !out) return record(DEM_ERR_INVALID_ARG, "%s", "dem_dsml_type: NULL argument");
    if (t >= d->s.types.size()) return record(DEM_ERR_INVALID_ARG, "no particle type %u", t);
    const PType& p = d->s.types[t];
    memset(out, 0, sizeof(*out));
    snprintf(out->id, sizeof(out->id), "%s", p.id.c_str());
    snprintf(out->name, sizeof(out->name), "%s", p.name.c_str());
    out->mass = p.mass;
    out->radius = p.radius;
    for (int c = 0; c < 3; ++c) out->color[c] = p.color[c];
    return DEM_OK;
}
