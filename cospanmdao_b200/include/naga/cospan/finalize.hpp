// naga/cospan/finalize.hpp — turning the recorded wiring into variables (Model::finalize).
//
// Every component port is a key (its path); a tie adds a key of its own. Connects and tie memberships join keys, and
// each joined set is one variable: one dtype, one rank, one device buffer. Promotions are names only (resolved by
// Runtime::resolve). Initializers and shape hooks attach to the variable their path names. The reference does the same
// bookkeeping in wiring.hpp:287-540 and model.hpp:733-754.
#pragma once

#include "model.hpp"

namespace naga::cospan {

inline void Model::finalize() {
    if (finalized_) return;
    if (!setup_done_) setup();
    auto& rt = *rt_;
    std::vector<System*> systems;
    std::function<void(System*)> walk = [&](System* s) {
        systems.push_back(s);
        for (auto& c : s->children_) {
            if (c->kind == Node::Kind::component) {
                rt.leaves.push_back(c.get());
                rt.components.push_back(static_cast<ComponentBase*>(c.get()));
            } else if (c->kind == Node::Kind::fused) {
                rt.leaves.push_back(c.get());
                auto* f = static_cast<FusedGroupBase*>(c.get());
                systems.push_back(f);
                for (auto* st : f->stages_) rt.components.push_back(st);
            } else {
                walk(static_cast<System*>(c.get()));
            }
        }
    };
    walk(root_.get());

    // union-find over keys
    std::map<std::string, int> ids;
    std::vector<std::string> keys;
    std::vector<int> up;
    auto key_id = [&](const std::string& k) {
        auto it = ids.find(k);
        if (it != ids.end()) return it->second;
        const int i = int(keys.size());
        ids[k] = i;
        keys.push_back(k);
        up.push_back(i);
        return i;
    };
    std::function<int(int)> find = [&](int i) { return up[i] == i ? i : (up[i] = find(up[i])); };
    auto unite = [&](const std::string& a, const std::string& b) {
        const int x = find(key_id(a)), y = find(key_id(b));
        if (x != y) up[y] = x;
    };
    struct PortRef {
        ComponentBase* c;
        detail::PortRec* p;
    };
    std::map<std::string, PortRef> port_of_key;
    for (ComponentBase* c : rt.components)
        for (auto& p : c->ports_) {
            const std::string k = c->path() + "." + p.name;
            key_id(k);
            port_of_key[k] = PortRef{c, &p};
        }
    struct TieRef {
        System* s;
        TieEntry t;
    };
    std::map<std::string, TieRef> tie_of_key;
    for (System* s : systems)
        for (auto& t : s->ties_) {
            const std::string k = s->path() + "/#" + t.name;
            if (tie_of_key.count(k))
                throw std::invalid_argument("naga::cospan: '" + s->path() + "' ties the name '" + t.name + "' twice");
            rt.tie_keys[s->path() + "/" + t.name] = k;
            key_id(k);
            tie_of_key[k] = TieRef{s, t};
        }
    for (System* s : systems) {
        for (auto& t : s->ties_) {
            if (t.members.size() < 2)
                throw std::invalid_argument("naga::cospan: the tie '" + t.name + "' in '" + s->path() + "' needs two members");
            for (auto& m : t.members) {
                const std::string mk = rt.resolve(s, m);
                auto pk = port_of_key.find(mk);
                if (pk != port_of_key.end()) {
                    if (pk->second.p->output != t.outputs)
                        throw std::invalid_argument("naga::cospan: the tie '" + t.name + "': '" + m + "' is " +
                                                    (t.outputs ? "an input" : "an output"));
                    if (t.outputs && t.policy == TieOutputsPolicy::require_atomic && !is_atomic(pk->second.p->dtype))
                        throw std::invalid_argument("naga::cospan: the tie '" + t.name + "' needs atomic outputs ('" + m +
                                                    "' is not)");
                }
                unite(s->path() + "/#" + t.name, mk);
            }
        }
        for (auto& [a, b] : s->connects_) {
            const std::string ka = rt.resolve(s, a), kb = rt.resolve(s, b);
            auto pa = port_of_key.find(ka), pb = port_of_key.find(kb);
            if (pb != port_of_key.end() && pb->second.p->output && (pa == port_of_key.end() || pa->second.p->output))
                throw std::invalid_argument("naga::cospan: connect('" + a + "', '" + b + "') in '" + s->path() +
                                            "': the destination is an output");
            unite(ka, kb);
        }
    }

    // variables
    std::map<int, int> var_of_root;
    auto var_for = [&](const std::string& k) -> detail::Var& {
        const int r = find(ids.at(k));
        auto it = var_of_root.find(r);
        if (it == var_of_root.end()) {
            detail::Var v;
            v.id = int(rt.vars.size());
            v.name = keys[r];
            var_of_root[r] = v.id;
            rt.vars.push_back(v);
            return rt.vars.back();
        }
        return rt.vars[it->second];
    };
    auto merge_spec = [](detail::Var& v, const ShapeSpec& s, const std::string& who) {
        if (s.empty()) return;
        if (v.spec.empty()) {
            v.spec = s;
            return;
        }
        for (int d = 0; d < s.rank && d < 4; ++d)
            if (s.known[d]) {
                if (v.spec.known[d] && v.spec.ext[d] != s.ext[d])
                    throw std::invalid_argument("naga::cospan: '" + who + "' declares dimension " + std::to_string(d) +
                                                " as " + std::to_string(s.ext[d]) + " but '" + v.name + "' has " +
                                                std::to_string(v.spec.ext[d]));
                v.spec.known[d] = true;
                v.spec.ext[d] = s.ext[d];
            }
    };
    for (auto& [k, pr] : port_of_key) {
        detail::Var& v = var_for(k);
        if (v.rank < 0) {
            v.rank = pr.p->rank;
            v.dtype = pr.p->dtype;
            v.name = k;
        } else if (v.rank != pr.p->rank || !dtype_compatible(v.dtype, pr.p->dtype)) {
            throw std::invalid_argument("naga::cospan: '" + k + "' (" + dtype_name(pr.p->dtype) + ", rank " +
                                        std::to_string(pr.p->rank) + ") is wired to '" + v.name + "' (" +
                                        dtype_name(v.dtype) + ", rank " + std::to_string(v.rank) + ")");
        }
        if (is_atomic(pr.p->dtype)) v.dtype = pr.p->dtype;
        if (pr.p->output) v.produced = true;
        if (pr.p->ragged) {
            v.ragged_port = true;
            if (pr.p->output) v.ragged_out = true;
            if (pr.p->counts) {
                if (v.declared_counts && *v.declared_counts != *pr.p->counts)
                    throw std::invalid_argument("naga::cospan: '" + k + "' declares the counts " + detail::list_of(*pr.p->counts) +
                                                " but '" + v.name + "' has " + detail::list_of(*v.declared_counts) +
                                                "; the counts must match");
                v.declared_counts = pr.p->counts;
            }
        }
        merge_spec(v, pr.p->declared, k);
        pr.p->var = v.id;
        rt.key_var[k] = v.id;
    }
    // a ragged output's variable is read by ragged ports only (a dense one cannot see per-index extents)
    for (auto& [k, pr] : port_of_key) {
        const detail::Var& v = rt.vars[pr.p->var];
        if (v.ragged_out && !pr.p->ragged)
            throw std::invalid_argument("naga::cospan: '" + k + "' reads the ragged variable '" + v.name +
                                        "'; a dense Input cannot see per-index extents (declare it as a RaggedInput)");
    }
    for (auto& [k, tr] : tie_of_key) {
        detail::Var& v = var_for(k);
        if (v.rank >= 0 && (v.rank != tr.t.rank || !dtype_compatible(v.dtype, tr.t.dtype)))
            throw std::invalid_argument("naga::cospan: the tie '" + tr.t.name + "' in '" + tr.s->path() +
                                        "' has another dtype or rank than its members");
        if (v.rank < 0) {
            v.rank = tr.t.rank;
            v.dtype = tr.t.dtype;
        }
        merge_spec(v, tr.t.shape, tr.s->path() + "." + tr.t.name);
        rt.key_var[k] = v.id;
    }

    // initializers: components' own, then systems' (later ones win, as a system initializes what it ties)
    for (ComponentBase* c : rt.components)
        for (auto& [name, init] : c->own_inits_) {
            auto* p = c->port(name);
            if (!p || p->output)
                throw std::invalid_argument("naga::cospan: '" + c->path() + "': init_input('" + name + "') names no input");
            detail::Var& v = rt.vars[p->var];
            v.init = init;
            v.stale = true;
        }
    for (System* s : systems)
        for (auto& [path, init] : s->inits_) {
            detail::Var& v = rt.var_of_path(s, path);
            v.init = init;
            v.stale = true;
        }
    for (System* s : systems)
        for (auto& h : s->hooks_) {
            detail::Var& v = rt.var_of_path(s, h.path);
            v.hook = h.dims;
            v.hook_sys = s;
            v.hook_path = s->path().empty() ? h.path : s->path() + "." + h.path;
        }
    detail::register_patterns(rt);
    finalized_ = true;
}

}  // namespace naga::cospan
