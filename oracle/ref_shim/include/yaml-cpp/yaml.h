// Oracle test infrastructure, not product code.
// Minimal stand-in for the part of yaml-cpp's Node that the reference's
// get_or (source/MosscapConfig.hpp) reads: a tree of named children with
// numeric leaves, so that the reference's own setup_gravity
// (source/SourceTerms/Gravity.cpp) can be called with a configuration built
// in code. No parsing.
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace YAML {

struct BadConversion : std::runtime_error {
    BadConversion() : std::runtime_error("bad conversion") {}
};

class Node {
public:
    Node() : tree_(std::make_shared<Tree>()) {}

    // Child `key`; an undefined Node when absent.
    Node operator[](const std::string& key) const {
        if (!tree_) {
            return Node(nullptr);
        }
        auto it = tree_->kids.find(key);
        if (it == tree_->kids.end()) {
            return Node(nullptr);
        }
        return it->second;
    }
    explicit operator bool() const { return tree_ && tree_->defined; }

    template <class T>
    T as() const {
        if (!tree_ || !tree_->is_value) {
            throw BadConversion();
        }
        return convert<T>();
    }

    // Building: child(key) creates the child; set(value) makes a leaf.
    Node child(const std::string& key) {
        auto it = tree_->kids.find(key);
        if (it != tree_->kids.end()) {
            return it->second;
        }
        Node n;
        tree_->kids.emplace(key, n);
        return n;
    }
    void set(double v) {
        tree_->is_value = true;
        tree_->value = v;
    }

private:
    struct Tree {
        bool defined = true;
        bool is_value = false;
        double value = 0.0;
        std::map<std::string, Node> kids;
    };
    explicit Node(std::nullptr_t) {}

    template <class T>
    T convert() const {
        if constexpr (std::is_same_v<T, std::string>) {
            return std::to_string(tree_->value);
        } else {
            return static_cast<T>(tree_->value);
        }
    }

    std::shared_ptr<Tree> tree_;
};

} // namespace YAML
