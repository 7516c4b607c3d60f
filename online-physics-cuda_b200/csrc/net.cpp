// The small nets a law declares (`net NAME in N hidden H... out M act A [file PATH]`): their starting weights and the
// weight files, in the reference's layout and text format (src/field/nn/Net.hpp, Net.cpp:241-333), so a trained file
// from the reference loads here unchanged.
#include "law.hpp"

#include <cmath>
#include <fstream>
#include <sstream>

namespace fe::law {

std::size_t NetDecl::weight_offset(int layer) const
{
    std::size_t at = 0;
    for (int l = 0; l < layer; ++l) {
        at += static_cast<std::size_t>(sizes[static_cast<std::size_t>(l)] + 1) * static_cast<std::size_t>(sizes[static_cast<std::size_t>(l) + 1]);
    }
    return at;
}

namespace {

// A 64-bit finalizer (the MurmurHash3 one): a well-spread word from a counter.
std::uint64_t finalize(std::uint64_t h)
{
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    return h;
}

} // namespace

void init_net(NetDecl& net, std::uint64_t seed)
{
    net.weights.assign(net.parameter_count(), 0.0f);
    std::uint64_t h = 1469598103934665603ull ^ seed; // FNV-1a of the name
    for (const char c : net.name) h = (h ^ static_cast<unsigned char>(c)) * 1099511628211ull;
    for (int l = 0; l + 1 < net.layers(); ++l) {
        const int ni = net.sizes[static_cast<std::size_t>(l)];
        const int no = net.sizes[static_cast<std::size_t>(l) + 1];
        const float limit = std::sqrt(6.0f / static_cast<float>(ni + no));
        float* w = net.weights.data() + net.weight_offset(l);
        for (int k = 0; k < ni * no; ++k) {
            const std::uint64_t r = finalize(h + static_cast<std::uint64_t>(l) * 0x9e3779b97f4a7c15ull + static_cast<std::uint64_t>(k));
            const float u = static_cast<float>(static_cast<double>(r >> 11) * (1.0 / 9007199254740992.0));
            w[k] = (2.0f * u - 1.0f) * limit;
        }
    }
    net.in_shift.assign(static_cast<std::size_t>(net.sizes.front()), 0.0f);
    net.in_scale.assign(static_cast<std::size_t>(net.sizes.front()), 1.0f);
    net.out_scale = 1.0f;
    net.loaded = false;
}

bool load_net(NetDecl& net, std::string& error)
{
    std::ifstream in(net.file);
    if (!in) {
        error = "no weights at " + net.file;
        return false;
    }
    std::vector<int> sizes;
    std::vector<float> shift, scale, weights;
    float out_scale = 1.0f;
    std::string act = net.act;
    std::string section, word;
    while (in >> word) {
        if (word == "net") {
            in >> word; // the name it was saved under
        } else if (word == "act") {
            in >> act;
            if (act != "tanh" && act != "relu" && act != "silu" && act != "linear") {
                error = net.file + ": unknown activation '" + act + "'";
                return false;
            }
            section.clear();
        } else if (word == "out_scale") {
            in >> out_scale;
            section.clear();
        } else if (word == "sizes" || word == "in_shift" || word == "in_scale" || word == "weights") {
            section = word;
        } else {
            std::istringstream number(word);
            double v = 0.0;
            if (!(number >> v)) {
                error = net.file + ": unexpected '" + word + "'";
                return false;
            }
            if (section == "sizes") sizes.push_back(static_cast<int>(v));
            else if (section == "in_shift") shift.push_back(static_cast<float>(v));
            else if (section == "in_scale") scale.push_back(static_cast<float>(v));
            else if (section == "weights") weights.push_back(static_cast<float>(v));
            else {
                error = net.file + ": a number outside any section";
                return false;
            }
        }
    }
    if (sizes != net.sizes) {
        error = net.file + ": its sizes are not the ones the law declares for '" + net.name + "'";
        return false;
    }
    if (act != net.act) {
        error = net.file + ": trained with another activation than the law declares";
        return false;
    }
    if (weights.size() != net.parameter_count()) {
        error = net.file + ": " + std::to_string(weights.size()) + " weights, the net has " + std::to_string(net.parameter_count());
        return false;
    }
    shift.resize(static_cast<std::size_t>(net.sizes.front()), 0.0f);
    scale.resize(static_cast<std::size_t>(net.sizes.front()), 1.0f);
    net.in_shift = std::move(shift);
    net.in_scale = std::move(scale);
    net.out_scale = out_scale;
    net.weights = std::move(weights);
    net.loaded = true;
    return true;
}

} // namespace fe::law
