// Banana particle data files (.bnn): see bnn_io.h for the layout.
#include "bnn_io.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <limits>
#include <sstream>

namespace bnnhost {

static void put(std::vector<unsigned char>& buf, const void* p, size_t n) {
    const unsigned char* c = (const unsigned char*)p;
    buf.insert(buf.end(), c, c + n);
}

void BnnFile::setFixedReal(const std::string& name, const float* v, uint32_t count) {
    Attribute a;
    a.type = "real";
    a.elementBytes = 4;
    a.count = count;
    put(a.data, v, sizeof(float) * count);
    fixed[name] = std::move(a);
}

void BnnFile::setFixedUInt(const std::string& name, const uint32_t* v, uint32_t count) {
    Attribute a;
    a.type = "uint";
    a.elementBytes = 4;
    a.count = count;
    put(a.data, v, sizeof(uint32_t) * count);
    fixed[name] = std::move(a);
}

void BnnFile::setParticleReal(const std::string& name, const float* v, uint32_t count) {
    Attribute a;
    a.type = "real";
    a.elementBytes = 4;
    a.count = count;
    put(a.data, v, sizeof(float) * count * (size_t)nParticles);
    particle[name] = std::move(a);
}

void BnnFile::setParticleCompressed(const std::string& name, const float* v, uint32_t count) {
    Attribute a;
    a.type = "compressed_real";
    a.elementBytes = 4;
    a.count = count;
    std::vector<float> lo(count, std::numeric_limits<float>::max()), hi(count, -std::numeric_limits<float>::max());
    for(size_t p = 0; p < nParticles; ++p)
        for(uint32_t c = 0; c < count; ++c) {
            const float x = v[p * count + c];
            lo[c] = x < lo[c] ? x : lo[c];
            hi[c] = x > hi[c] ? x : hi[c];
        }
    if(nParticles == 0)
        for(uint32_t c = 0; c < count; ++c) lo[c] = hi[c] = 0.f;
    put(a.data, lo.data(), sizeof(float) * count);
    put(a.data, hi.data(), sizeof(float) * count);
    std::vector<uint16_t> q((size_t)nParticles * count);
    for(size_t p = 0; p < nParticles; ++p)
        for(uint32_t c = 0; c < count; ++c) {
            const float diff = hi[c] - lo[c];
            q[p * count + c] = diff > 0.f ? (uint16_t)(65535.0f * ((v[p * count + c] - lo[c]) / diff)) : (uint16_t)0;
        }
    put(a.data, q.data(), sizeof(uint16_t) * q.size());
    particle[name] = std::move(a);
}

void BnnFile::setParticleCompressedMatrix(const std::string& name, const float* v, uint32_t dim) {
    Attribute a;
    a.type = "compressed_real";
    a.elementBytes = 4;
    a.count = dim * dim;
    const size_t total = (size_t)nParticles * a.count;
    float lo = std::numeric_limits<float>::max(), hi = -std::numeric_limits<float>::max();
    for(size_t i = 0; i < total; ++i) {
        lo = v[i] < lo ? v[i] : lo;
        hi = v[i] > hi ? v[i] : hi;
    }
    if(total == 0) lo = hi = 0.f;
    put(a.data, &lo, sizeof(float));
    put(a.data, &hi, sizeof(float));
    const float diff = hi - lo;
    std::vector<uint16_t> q(total);
    for(size_t i = 0; i < total; ++i) q[i] = diff > 0.f ? (uint16_t)(65535.0f * ((v[i] - lo) / diff)) : (uint16_t)0;
    put(a.data, q.data(), sizeof(uint16_t) * q.size());
    particle[name] = std::move(a);
}

void BnnFile::setParticleUInt16(const std::string& name, const uint16_t* v) {
    Attribute a;
    a.type = "uint16";
    a.elementBytes = 2;
    a.count = 1;
    put(a.data, v, sizeof(uint16_t) * (size_t)nParticles);
    particle[name] = std::move(a);
}

bool BnnFile::write(const std::string& path) const {
    std::ofstream f(path, std::ios::binary | std::ios::out);
    if(!f) return false;
    f.imbue(std::locale("C"));
    f << "BananaParticleData\n";
    for(const auto& kv : fixed)
        f << "FixedAttribute " << kv.first << " " << kv.second.type << " " << kv.second.elementBytes << " "
          << kv.second.count << " " << kv.second.data.size() << "\n";
    for(const auto& kv : particle)
        f << "ParticleAttribute " << kv.first << " " << kv.second.type << " " << kv.second.elementBytes << " "
          << kv.second.count << " " << kv.second.data.size() << "\n";
    f << "NParticles " << nParticles << "\n";
    f << "EndHeader.\n";
    for(const auto& kv : fixed) f.write((const char*)kv.second.data.data(), (std::streamsize)kv.second.data.size());
    for(const auto& kv : particle) f.write((const char*)kv.second.data.data(), (std::streamsize)kv.second.data.size());
    return (bool)f;
}

bool BnnFile::read(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if(!f) return false;
    fixed.clear();
    particle.clear();
    nParticles = 0;
    std::string line;
    if(!std::getline(f, line) || line != "BananaParticleData") return false;
    std::vector<std::pair<bool, std::string>> order;  // (is fixed, name) in header order
    for(;;) {
        if(!std::getline(f, line)) return false;
        if(line == "EndHeader.") break;
        std::istringstream ss(line);
        ss.imbue(std::locale("C"));
        std::string kind;
        ss >> kind;
        if(kind == "NParticles") {
            ss >> nParticles;
            continue;
        }
        if(kind != "FixedAttribute" && kind != "ParticleAttribute") return false;
        std::string name;
        Attribute a;
        size_t bytes = 0;
        ss >> name >> a.type >> a.elementBytes >> a.count >> bytes;
        if(!ss) return false;
        a.data.resize(bytes);
        const bool isFixed = kind == "FixedAttribute";
        (isFixed ? fixed : particle)[name] = std::move(a);
        order.emplace_back(isFixed, name);
    }
    for(const auto& o : order) {
        Attribute& a = (o.first ? fixed : particle)[o.second];
        if(!f.read((char*)a.data.data(), (std::streamsize)a.data.size())) return false;
    }
    return true;
}

static const BnnFile::Attribute* find(const BnnFile& b, const std::string& name) {
    auto it = b.particle.find(name);
    if(it != b.particle.end()) return &it->second;
    auto jt = b.fixed.find(name);
    return jt != b.fixed.end() ? &jt->second : nullptr;
}

bool BnnFile::getFloats(const std::string& name, std::vector<float>& out) const {
    const Attribute* a = find(*this, name);
    if(!a) return false;
    if(a->type == "real" && a->elementBytes == 4) {
        out.resize(a->data.size() / 4);
        std::memcpy(out.data(), a->data.data(), a->data.size());
        return true;
    }
    if(a->type == "compressed_real") {
        const uint32_t c = a->count;
        const float* lo = (const float*)a->data.data();
        const float* hi = lo + c;
        const uint16_t* q = (const uint16_t*)(a->data.data() + 8 * (size_t)c);
        const size_t n = (a->data.size() - 8 * (size_t)c) / 2;
        out.resize(n);
        // ParticleHelpers::decompress (ParticleHelpers.cpp:183-199)
        for(size_t i = 0; i < n; ++i) out[i] = (float)q[i] * (hi[i % c] - lo[i % c]) / 65535.0f + lo[i % c];
        return true;
    }
    return false;
}

bool BnnFile::getMatrixFloats(const std::string& name, std::vector<float>& out) const {
    const Attribute* a = find(*this, name);
    if(!a) return false;
    if(a->type == "real" && a->elementBytes == 4) return getFloats(name, out);
    if(a->type != "compressed_real" || a->data.size() < 8) return false;
    float lo, hi;
    std::memcpy(&lo, a->data.data(), 4);
    std::memcpy(&hi, a->data.data() + 4, 4);
    const uint16_t* q = (const uint16_t*)(a->data.data() + 8);
    const size_t n = (a->data.size() - 8) / 2;
    out.resize(n);
    // ParticleHelpers::decompress for matrices (ParticleHelpers.cpp:234-252)
    const float diff = hi - lo;
    for(size_t i = 0; i < n; ++i) out[i] = (float)q[i] * diff / 65535.0f + lo;
    return true;
}

bool BnnFile::getUInts(const std::string& name, std::vector<uint32_t>& out) const {
    const Attribute* a = find(*this, name);
    if(!a || a->elementBytes != 4) return false;
    out.resize(a->data.size() / 4);
    std::memcpy(out.data(), a->data.data(), a->data.size());
    return true;
}

bool BnnFile::getUInt16(const std::string& name, std::vector<uint16_t>& out) const {
    const Attribute* a = find(*this, name);
    if(!a || a->elementBytes != 2) return false;
    out.resize(a->data.size() / 2);
    std::memcpy(out.data(), a->data.data(), a->data.size());
    return true;
}

std::string bnn_file_path(const std::string& root, const std::string& folder, const std::string& name, int id) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), ".%04d.bnn", id);
    return root + "/" + folder + "/" + name + buf;
}

// FileHelpers::createFolder (FileHelpers.h:43-53) creates every missing folder of the
// path ("mkdir -p"); so does this
bool make_output_folder(const std::string& root, const std::string& folder) {
    const std::string p = root + "/" + folder;
    std::error_code ec;
    std::filesystem::create_directories(p, ec);
    return std::filesystem::is_directory(p, ec);
}

} // namespace bnnhost
