from .tensorcircuit import TensorCircuit, compile
