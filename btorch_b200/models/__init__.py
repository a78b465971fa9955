"""Module API of btorch.models for the recurrent spiking step."""

from . import cudagraph, environ, functional
from .cudagraph import CudaGraphRunner
from .base import BaseNode, MemoryModule, ParamBufferMixin, StepModule
from .history import SpikeHistory
from .constrain import HasConstraint, constrain_net
from .linear import BaseSparseConn, DenseConn, SparseConn, SparseConstrainedConn
from .neurons import ALIF, LIF
from .rnn import RecurrentNN, RecurrentNNAbstract, make_rnn
from .surrogate import Sigmoid
from .synapse import BasePSC, DelayedPSC, ExponentialPSC, HeterSynapsePSC

__all__ = ["cudagraph", "CudaGraphRunner", "environ", "functional", "BaseNode", "MemoryModule", "ParamBufferMixin", "StepModule", "SpikeHistory",
           "BaseSparseConn", "DenseConn", "SparseConn", "SparseConstrainedConn", "HasConstraint", "constrain_net", "ALIF", "LIF", "RecurrentNN", "RecurrentNNAbstract",
           "make_rnn", "Sigmoid", "BasePSC", "DelayedPSC", "ExponentialPSC", "HeterSynapsePSC"]
