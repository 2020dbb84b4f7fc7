// The closed Tecplot TECIO library is absent from this image. The reference
// calls it only to write and read .plt visualisation files; every call becomes a
// no-op returning 0. No arithmetic of the solver passes through these calls.
#pragma once
#include <cstdint>
typedef int INTEGER4;
typedef enum { FieldDataType_Reserved = 0, FieldDataType_Float, FieldDataType_Double,
               FieldDataType_Int32, FieldDataType_Int16, FieldDataType_Byte,
               FieldDataType_Bit, FieldDataType_Int64 } FieldDataType_e;
#define FieldDataType_Int FieldDataType_Int32
#define PLFBS_TEC_STUB(fn) template <typename... A> static inline int fn(A...) { return 0; }
PLFBS_TEC_STUB(TECAUXSTR142) PLFBS_TEC_STUB(TECDAT142) PLFBS_TEC_STUB(TECEND142)
PLFBS_TEC_STUB(TECINI142) PLFBS_TEC_STUB(TECNODE142) PLFBS_TEC_STUB(TECZNE142)
PLFBS_TEC_STUB(tecDataSetGetNumVars) PLFBS_TEC_STUB(tecDataSetGetNumZones)
PLFBS_TEC_STUB(tecDataSetGetTitle) PLFBS_TEC_STUB(tecFileGetType)
PLFBS_TEC_STUB(tecFileReaderOpen) PLFBS_TEC_STUB(tecStringFree) PLFBS_TEC_STUB(tecVarGetName)
PLFBS_TEC_STUB(tecZoneAddAuxData) PLFBS_TEC_STUB(tecZoneAuxDataGetItem)
PLFBS_TEC_STUB(tecZoneAuxDataGetNumItems) PLFBS_TEC_STUB(tecZoneConnectivityGetSharedZone)
PLFBS_TEC_STUB(tecZoneFaceNbrGetConnections) PLFBS_TEC_STUB(tecZoneFaceNbrGetConnections64)
PLFBS_TEC_STUB(tecZoneFaceNbrGetMode) PLFBS_TEC_STUB(tecZoneFaceNbrGetNumConnections)
PLFBS_TEC_STUB(tecZoneFaceNbrGetNumValues) PLFBS_TEC_STUB(tecZoneFaceNbrWriteConnections32)
PLFBS_TEC_STUB(tecZoneFaceNbrWriteConnections64) PLFBS_TEC_STUB(tecZoneFaceNbrsAre64Bit)
PLFBS_TEC_STUB(tecZoneGetIJK) PLFBS_TEC_STUB(tecZoneGetParentZone)
PLFBS_TEC_STUB(tecZoneGetSolutionTime) PLFBS_TEC_STUB(tecZoneGetStrandID)
PLFBS_TEC_STUB(tecZoneGetTitle) PLFBS_TEC_STUB(tecZoneGetType)
PLFBS_TEC_STUB(tecZoneNodeMapGet) PLFBS_TEC_STUB(tecZoneNodeMapGet64)
PLFBS_TEC_STUB(tecZoneNodeMapGetNumValues) PLFBS_TEC_STUB(tecZoneNodeMapIs64Bit)
PLFBS_TEC_STUB(tecZoneNodeMapWrite32) PLFBS_TEC_STUB(tecZoneNodeMapWrite64)
PLFBS_TEC_STUB(tecZoneVarGetDoubleValues) PLFBS_TEC_STUB(tecZoneVarGetFloatValues)
PLFBS_TEC_STUB(tecZoneVarGetInt16Values) PLFBS_TEC_STUB(tecZoneVarGetInt32Values)
PLFBS_TEC_STUB(tecZoneVarGetNumValues) PLFBS_TEC_STUB(tecZoneVarGetSharedZone)
PLFBS_TEC_STUB(tecZoneVarGetType) PLFBS_TEC_STUB(tecZoneVarGetUInt8Values)
PLFBS_TEC_STUB(tecZoneVarGetValueLocation) PLFBS_TEC_STUB(tecZoneVarIsPassive)
PLFBS_TEC_STUB(tecZoneVarWriteDoubleValues) PLFBS_TEC_STUB(tecZoneVarWriteFloatValues)
PLFBS_TEC_STUB(tecZoneVarWriteInt16Values) PLFBS_TEC_STUB(tecZoneVarWriteInt32Values)
PLFBS_TEC_STUB(tecZoneVarWriteUInt8Values) PLFBS_TEC_STUB(tecpolyface142)
#undef PLFBS_TEC_STUB
