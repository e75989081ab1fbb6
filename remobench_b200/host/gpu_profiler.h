// Named GPU time scopes (include/remo/GpuProfiler.h), fed with device times
// the C ABI measures with CUDA events on the launching stream.
#pragma once

#include <algorithm>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace rbhost {

struct ScopeStats {
    std::vector<double> samples;  // ms, one per launch of the scope
    double total() const {
        double t = 0.0;
        for (double s : samples) t += s;
        return t;
    }
    uint64_t count() const { return samples.size(); }
    double last() const { return samples.empty() ? 0.0 : samples.back(); }
    double min() const { return samples.empty() ? 0.0 : *std::min_element(samples.begin(), samples.end()); }
    double max() const { return samples.empty() ? 0.0 : *std::max_element(samples.begin(), samples.end()); }
    // Nearest-rank percentile, q in [0, 1].
    double percentile(double q) const {
        if (samples.empty()) return 0.0;
        std::vector<double> s(samples);
        std::sort(s.begin(), s.end());
        const size_t k = static_cast<size_t>(std::min<double>(s.size() - 1, q * (s.size() - 1) + 0.5));
        return s[k];
    }
    double median() const { return percentile(0.5); }
};

class GpuProfiler {
public:
    void addSample(const std::string& name, double ms) {
        auto it = m_scopes.find(name);
        if (it == m_scopes.end()) {
            m_order.push_back(name);
            it = m_scopes.emplace(name, ScopeStats{}).first;
        }
        it->second.samples.push_back(ms);
    }
    const ScopeStats* find(const std::string& name) const {
        auto it = m_scopes.find(name);
        return it == m_scopes.end() ? nullptr : &it->second;
    }
    // Drops every scope whose name starts with prefix (a pipeline's reset).
    void clearPrefix(const std::string& prefix) {
        for (auto it = m_scopes.begin(); it != m_scopes.end();) {
            if (it->first.compare(0, prefix.size(), prefix) == 0)
                it = m_scopes.erase(it);
            else
                ++it;
        }
        m_order.erase(std::remove_if(m_order.begin(), m_order.end(),
                                     [&](const std::string& n) { return n.compare(0, prefix.size(), prefix) == 0; }),
                      m_order.end());
    }
    // Scope names in order of first sample.
    const std::vector<std::string>& scopeNames() const { return m_order; }

private:
    std::map<std::string, ScopeStats> m_scopes;
    std::vector<std::string> m_order;
};

}  // namespace rbhost
