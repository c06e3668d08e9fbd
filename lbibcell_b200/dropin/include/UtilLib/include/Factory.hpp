// UtilLib::Factory (libs/UtilLib/include/Factory.hpp:105-160): creators
// registered by name; createObject of an unknown name throws std::bad_typeid
// (ErrorPolicyThrowException, :45-47), as plugin registries expect.
#ifndef LBIBCELL_DROPIN_UTILLIB_FACTORY_HPP
#define LBIBCELL_DROPIN_UTILLIB_FACTORY_HPP

#include <map>
#include <typeinfo>

namespace UtilLib {

template <typename IdentifierType, typename ProductType>
class ErrorPolicyThrowException {
 protected:
    static ProductType* onUnknownType(const IdentifierType&) { throw std::bad_typeid(); }
};

template <typename IdentifierType, typename ProductType>
class ErrorPolicyReturnNull {
 protected:
    static ProductType* onUnknownType(const IdentifierType&) { return 0; }
};

template <class AbstractProduct, typename IdentifierType,
          template <typename, class> class FactoryErrorPolicy = ErrorPolicyThrowException,
          typename ProductCreatorSignature = AbstractProduct* (*)()>
class Factory : public FactoryErrorPolicy<IdentifierType, AbstractProduct> {
 public:
    bool registerType(const IdentifierType& id, ProductCreatorSignature creator) {
        return creators_.insert(std::make_pair(id, creator)).second;
    }
    bool unregisterType(const IdentifierType& id) { return creators_.erase(id) == 1; }
    bool isRegistered(const IdentifierType& id) const { return creators_.count(id) != 0; }
    AbstractProduct* createObject(const IdentifierType& id) const {
        typename std::map<IdentifierType, ProductCreatorSignature>::const_iterator it = creators_.find(id);
        if (it != creators_.end()) return (it->second)();
        return this->onUnknownType(id);
    }

 private:
    std::map<IdentifierType, ProductCreatorSignature> creators_;
};

}  // namespace UtilLib

#endif
