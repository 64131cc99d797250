// Test infrastructure only: stand-in for the external `VectorMap` container that the
// reference's DataBase.cpp uses (DataBase.cpp:26,96,151-165,170-174).  Semantics taken from
// those use sites: `map[key]` default-inserts, iteration visits values (insertion order),
// `getKey(valueRef)` maps a value reference obtained from iteration back to its key, and
// `clear/empty/size`.
#pragma once
#include <cstddef>
#include <cstdint>
#include <unordered_map>
#include <vector>

template <typename Key, typename Value>
class VectorMap
{
public:
    Value& operator[](const Key& key)
    {
        const auto it = mIndex.find(key);
        if (it != mIndex.end()) {
            return mValues[it->second];
        }
        mIndex.emplace(key, mValues.size());
        mKeys.push_back(key);
        mValues.emplace_back();
        return mValues.back();
    }
    Key getKey(const Value& ref) const { return mKeys.at(static_cast<size_t>(&ref - mValues.data())); }
    typename std::vector<Value>::iterator begin() { return mValues.begin(); }
    typename std::vector<Value>::iterator end() { return mValues.end(); }
    typename std::vector<Value>::const_iterator begin() const { return mValues.begin(); }
    typename std::vector<Value>::const_iterator end() const { return mValues.end(); }
    size_t size() const { return mValues.size(); }
    bool empty() const { return mValues.empty(); }
    void clear()
    {
        mValues.clear();
        mKeys.clear();
        mIndex.clear();
    }

private:
    std::vector<Value> mValues;
    std::vector<Key> mKeys;
    std::unordered_map<Key, size_t> mIndex;
};
