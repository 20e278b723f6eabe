// Banana particle data files (.bnn): the reference's ParticleSerialization container
// (Simulation/ParticleTools/ParticleSerialization.h:32-212, .cpp:479-632), written and read
// with the same header, attribute types and encodings so files move between the reference
// tools and this solver.
//
//   "BananaParticleData\n"
//   "FixedAttribute <name> <type> <elementBytes> <count> <dataBytes>\n"      (name order)
//   "ParticleAttribute <name> <type> <elementBytes> <count> <dataBytes>\n"   (name order)
//   "NParticles <n>\n"
//   "EndHeader.\n"
//   <data of the fixed attributes, then of the particle attributes, in header order>
//
// Types used by the fluid solvers: "real" (raw float), "uint" (raw uint32), "uint16", and
// "compressed_real": float min[count], float max[count], then one uint16 per component,
// trunc(65535 * (v - min) / (max - min)) (ParticleHelpers.cpp:46-80; a component whose
// max equals its min is stored as 0).  A matrix attribute ("anisotropic_kernel", count 9)
// is compressed with one min and one max over all its entries (ParticleHelpers.cpp:82-114).
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace bnnhost {

class BnnFile {
public:
    struct Attribute {
        std::string type;            // "real", "uint", "uint16", "compressed_real", ...
        uint32_t elementBytes = 4;
        uint32_t count = 1;          // components per value
        std::vector<unsigned char> data;
    };

    uint32_t nParticles = 0;
    std::map<std::string, Attribute> fixed;
    std::map<std::string, Attribute> particle;

    // ---- writing
    void setFixedReal(const std::string& name, const float* v, uint32_t count);
    void setFixedUInt(const std::string& name, const uint32_t* v, uint32_t count);
    void setParticleReal(const std::string& name, const float* v, uint32_t count);       // nParticles x count
    void setParticleCompressed(const std::string& name, const float* v, uint32_t count); // nParticles x count
    void setParticleCompressedMatrix(const std::string& name, const float* v, uint32_t dim);  // nParticles x dim^2
    void setParticleUInt16(const std::string& name, const uint16_t* v);
    bool write(const std::string& path) const;

    // ---- reading
    bool read(const std::string& path);
    // Raw floats of a "real" attribute, or the decoded values of a "compressed_real" one
    bool getFloats(const std::string& name, std::vector<float>& out) const;
    // Decoded values of a matrix attribute (compressed with one min / max for all entries)
    bool getMatrixFloats(const std::string& name, std::vector<float>& out) const;
    bool getUInts(const std::string& name, std::vector<uint32_t>& out) const;
    bool getUInt16(const std::string& name, std::vector<uint16_t>& out) const;
};

// DataIO::getFilePath (Data/DataIO.h:119-124): <root>/<folder>/<name>.<4-digit id>.bnn
std::string bnn_file_path(const std::string& root, const std::string& folder, const std::string& name, int id);
// Creates <root>/<folder> (and <root>) when missing
bool make_output_folder(const std::string& root, const std::string& folder);

} // namespace bnnhost
